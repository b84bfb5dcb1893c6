"""Build libnabla_b200.so in-tree for sm_100a (B200).

    python nabla-ai_b200/build.py [--debug]

Compiles every CUDA/C++ source in csrc/ with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into nabla-ai_b200/lib/.
Object files go to nabla-ai_b200/_build/. Sources are rebuilt only when
they (or a header) changed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libnabla_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-Wall", "-I" + CSRC, "-I" + os.path.join(REPO, "include")]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit(f"build failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    newest_hdr = max(os.path.getmtime(h) for h in hdrs)
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if os.path.exists(o) and os.path.getmtime(o) > max(os.path.getmtime(s), newest_hdr):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, *(extra or []), "-x", "cu", "-c", "-o", o, s]
        out = _run(cmd)
        if verbose and out.strip():
            print(out)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
