"""nabla_b200 — host-side Python mirror of the reference's solver interface over
the C ABI in include/nabla_b200.h (ctypes). The compute path is the CUDA library."""
from . import abi, cases  # noqa: F401
