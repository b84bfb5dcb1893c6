"""The C-ABI library loads, exports every declared symbol, and fails loudly
(no CPU fallback) where no sm_100 GPU is present. CPU only."""
import ctypes as C
import os

import pytest

from nabla_b200 import abi


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    declared = abi.declared_symbols()
    assert len(declared) >= 19
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # the ctypes prototype table covers the header
    assert sorted(n for n, _, _ in abi.PROTOTYPES) == declared


def test_status_strings():
    lib = abi.load()
    assert lib.nb_status_string(abi.NB_OK) == b"ok"
    assert lib.nb_status_string(abi.NB_ERR_CUDA) == b"CUDA error"


def test_struct_layouts_match_header():
    # sizes implied by include/nabla_b200.h on LP64
    assert C.sizeof(abi.FaceBC) == 48
    assert C.sizeof(abi.GridDesc) == 16 + 24 + 24 + 6 * 48 + 8
    assert C.sizeof(abi.StepReport) == 8 + 10 * 8 + 8 + 8


def test_no_gpu_means_error_not_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = abi.load()
    h = C.c_void_p()
    assert lib.nb_ctx_create(0, C.byref(h)) == abi.NB_ERR_CUDA
    assert not h.value


def test_library_links_no_oracle():
    """The product library must not depend on the oracle libraries."""
    import subprocess
    out = subprocess.run(["ldd", abi.LIB_PATH], capture_output=True, text=True).stdout
    assert "orc" not in out and "nabla_ref" not in out
    assert os.path.basename(abi.LIB_PATH) == "libnabla_b200.so"


def test_cpp_header_compiles_against_c_abi(tmp_path):
    """include/nabla_b200.hpp (the C++20 host API) compiles and links against the library."""
    import subprocess
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "use.cpp"
    src.write_text('#include "nabla_b200.hpp"\n'
                   'int main() { try { auto c = std::make_shared<nabla_b200::Context>(0);'
                   ' nabla_b200::MgPoisson mg(c); return mg.name().empty(); }'
                   ' catch (const nabla_b200::Error& e) { return e.status() == NB_ERR_CUDA ? 0 : 2; } }\n')
    exe = tmp_path / "use"
    r = subprocess.run(["g++", "-std=c++20", "-I", os.path.join(repo, "include"), str(src), "-o", str(exe),
                        "-L", os.path.dirname(abi.LIB_PATH), "-lnabla_b200",
                        "-Wl,-rpath," + os.path.dirname(abi.LIB_PATH)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([str(exe)]).returncode == 0
