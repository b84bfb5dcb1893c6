"""TEST INFRASTRUCTURE ONLY — Python access to the two CPU oracles.

* ``Restatement``: this repo's plain-C restatement (oracle/_build/liborc.so).
* ``Reference``: the reference's own CPU code compiled in place
  (oracle/_ref/libnabla_ref.so, built by oracle/Makefile from the reference tree).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg import
this module. The product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "nabla-ai_b200"))
from nabla_b200 import abi  # noqa: E402  (struct layouts shared with the C ABI header)

ORC_PATH = os.path.join(HERE, "_build", "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "libnabla_ref.so")
DROPIN_PATH = os.path.join(HERE, "_ref", "libnabla_dropin.so")

GP = C.POINTER(abi.GridDesc)
FP = C.POINTER(abi.FlowConfig)
DP = abi.DP
RP = C.POINTER(abi.StepReport)
PRP = C.POINTER(abi.PoissonReport)


def _load(path):
    if not os.path.exists(path):
        raise RuntimeError(f"oracle library {path} missing; run `make -C oracle`")
    return C.CDLL(path)


class _Common:
    """Shared Python wrappers over a library exposing <prefix>_ entry points."""

    def apply_a(self, grid, x):
        out = np.zeros(grid.ncell)
        self._apply_a(C.byref(grid.desc()), abi.dptr(np.ascontiguousarray(x, dtype=np.float64)),
                      abi.dptr(out))
        return out

    def poisson(self, grid, b, tol, maxit, kind="mg"):
        x = np.zeros(grid.ncell)
        rep = abi.PoissonReport()
        self._solve(kind, grid, np.ascontiguousarray(b, dtype=np.float64), x, tol, maxit, rep)
        return x, rep


class Restatement(_Common):
    def __init__(self, path=ORC_PATH):
        L = self.lib = _load(path)
        L.orc_apply_a.argtypes = [GP, DP, DP]
        L.orc_build_diagonal.argtypes = [GP, DP]
        L.orc_cg_solve.argtypes = [GP, DP, DP, C.c_double, C.c_int, PRP]
        L.orc_mg_solve.argtypes = [GP, DP, DP, C.c_double, C.c_int, PRP]
        L.orc_ns_create.restype = C.c_void_p
        L.orc_ns_create.argtypes = [GP, FP]
        L.orc_ns_destroy.argtypes = [C.c_void_p]
        L.orc_ns_initialize.argtypes = [C.c_void_p]
        L.orc_ns_set_state.argtypes = [C.c_void_p, DP, DP, DP, DP, C.c_int, C.c_double, C.c_double]
        L.orc_ns_get_state.argtypes = [C.c_void_p, DP, DP, DP, DP]
        L.orc_ns_compute_dt.restype = C.c_double
        L.orc_ns_compute_dt.argtypes = [C.c_void_p]
        L.orc_ns_step.argtypes = [C.c_void_p, C.c_double, RP]
        L.orc_morton_encode.restype = C.c_uint64
        L.orc_morton_encode.argtypes = [C.c_uint32] * 3
        L.orc_morton_decode.argtypes = [C.c_uint64] + [C.POINTER(C.c_uint32)] * 3
        self._apply_a = L.orc_apply_a

    def _solve(self, kind, grid, b, x, tol, maxit, rep):
        fn = self.lib.orc_mg_solve if kind == "mg" else self.lib.orc_cg_solve
        fn(C.byref(grid.desc()), abi.dptr(b), abi.dptr(x), tol, maxit, C.byref(rep))

    def ns(self, grid, cfg):
        return _NS(self.lib, "orc", grid, cfg)

    def amr(self, geom, leaves, cfg, solid=None):
        return AmrStep(self.lib, geom, leaves, cfg, solid)

    def morton_encode(self, x, y, z):
        return self.lib.orc_morton_encode(x, y, z)


class AmrStep:
    """The oracle's octree MAC step (oracle/restate_amr.c). Faces and cells are
    addressed by (level, i, j, k) index arrays, as AmrCase.face_index and
    amr.cell_coords produce them."""

    def __init__(self, lib, geom, leaves, cfg, solid=None):
        self.lib = lib
        I32 = C.POINTER(C.c_int32)
        lib.orc_amr_create.restype = C.c_void_p
        lib.orc_amr_create.argtypes = [C.POINTER(abi.AmrGeom), I32, C.c_int64, C.POINTER(C.c_uint8), FP]
        lib.orc_amr_destroy.argtypes = [C.c_void_p]
        lib.orc_amr_set.argtypes = [C.c_void_p, C.c_int, C.c_int64, I32, I32, I32, I32, DP]
        lib.orc_amr_get.argtypes = [C.c_void_p, C.c_int, C.c_int64, I32, I32, I32, I32, DP]
        lib.orc_amr_step.restype = C.c_double
        lib.orc_amr_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_int)]
        self._leaves = np.ascontiguousarray(leaves, dtype=np.int32)
        sp = None
        if solid is not None:
            self._solid = np.ascontiguousarray(solid, dtype=np.uint8)
            sp = self._solid.ctypes.data_as(C.POINTER(C.c_uint8))
        self._cfg = cfg
        self.h = lib.orc_amr_create(C.byref(geom), self._leaves.ctypes.data_as(I32), self._leaves.shape[0], sp,
                                    C.byref(cfg))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_amr_destroy(self.h)
            self.h = None

    @staticmethod
    def _idx(ix):
        return [np.ascontiguousarray(a, dtype=np.int32) for a in ix]

    def set(self, comp, index, values):
        lev, i, j, k = self._idx(index)
        v = np.ascontiguousarray(values, dtype=np.float64)
        P = C.POINTER(C.c_int32)
        self.lib.orc_amr_set(self.h, comp, v.size, lev.ctypes.data_as(P), i.ctypes.data_as(P), j.ctypes.data_as(P),
                             k.ctypes.data_as(P), abi.dptr(v))

    def get(self, comp, index):
        lev, i, j, k = self._idx(index)
        out = np.zeros(lev.size)
        P = C.POINTER(C.c_int32)
        self.lib.orc_amr_get(self.h, comp, lev.size, lev.ctypes.data_as(P), i.ctypes.data_as(P), j.ctypes.data_as(P),
                             k.ctypes.data_as(P), abi.dptr(out))
        return out

    def step(self, dt, tol=1e-13):
        it = C.c_int()
        dmax = self.lib.orc_amr_step(self.h, dt, tol, C.byref(it))
        return dmax, it.value


class Reference(_Common):
    def __init__(self, path=REF_PATH):
        L = self.lib = _load(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_apply_a.argtypes = [GP, DP, DP]
        L.ref_build_diagonal.argtypes = [GP, DP]
        L.ref_poisson_solve.argtypes = [C.c_int, GP, DP, DP, C.c_double, C.c_int, PRP]
        L.ref_ns_create.restype = C.c_void_p
        L.ref_ns_create.argtypes = [GP, FP]
        L.ref_ns_destroy.argtypes = [C.c_void_p]
        L.ref_ns_initialize.argtypes = [C.c_void_p]
        L.ref_ns_set_state.argtypes = [C.c_void_p, DP, DP, DP, DP, C.c_int, C.c_double, C.c_double]
        L.ref_ns_get_state.argtypes = [C.c_void_p, DP, DP, DP, DP]
        L.ref_ns_compute_dt.restype = C.c_double
        L.ref_ns_compute_dt.argtypes = [C.c_void_p]
        L.ref_ns_step.argtypes = [C.c_void_p, C.c_double, RP]
        L.ref_ns_write_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_ns_read_checkpoint.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_run_case.argtypes = [GP, FP, C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_char_p,
                                   DP, C.POINTER(C.c_int)]
        L.ref_load_case.argtypes = [C.c_char_p, GP, C.POINTER(C.c_uint8), C.c_uint64, FP, C.c_char_p, C.c_int,
                                    C.POINTER(C.c_int), DP]
        L.ref_morton_encode.restype = C.c_uint64
        L.ref_morton_encode.argtypes = [C.c_uint32] * 3
        L.ref_morton_decode.argtypes = [C.c_uint64] + [C.POINTER(C.c_uint32)] * 3
        L.ref_make_case.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, GP,
                                    C.POINTER(C.c_uint8), FP]
        L.ref_octree_create.restype = C.c_void_p
        L.ref_octree_create.argtypes = [DP, DP, C.c_int]
        L.ref_octree_destroy.argtypes = [C.c_void_p]
        L.ref_octree_refine_uniform.argtypes = [C.c_void_p, C.c_int]
        L.ref_octree_refine_box.argtypes = [C.c_void_p, DP, DP, C.c_int]
        L.ref_octree_refine_morton.argtypes = [C.c_void_p, C.c_uint64]
        L.ref_octree_coarsen.argtypes = [C.c_void_p, C.c_uint64, C.c_int]
        L.ref_octree_is_balanced.argtypes = [C.c_void_p]
        L.ref_octree_cell_count.restype = C.c_uint64
        L.ref_octree_cell_count.argtypes = [C.c_void_p]
        L.ref_octree_cells.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint8),
                                       C.POINTER(C.c_uint8)]
        L.ref_octree_set_mask.argtypes = [C.c_void_p, C.c_uint64, C.c_int]
        L.ref_octree_cell_center.argtypes = [C.c_void_p, C.c_uint64, DP]
        L.ref_octree_face_neighbors.argtypes = [C.c_void_p, C.c_uint64, C.c_int,
                                                C.POINTER(C.c_uint64)]
        L.ref_octree_apply_a.argtypes = [C.c_void_p, DP, DP]
        L.ref_octree_build_diagonal.argtypes = [C.c_void_p, DP]
        L.ref_octree_solve.argtypes = [C.c_void_p, DP, DP, C.c_double, C.c_int, PRP]
        L.ref_uniform.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_uint64, DP]
        self._apply_a = L.ref_apply_a

    def uniform(self, seed, n, lo=-1.0, hi=1.0, bits64=False):
        """n draws of std::uniform_real_distribution(lo, hi) over mt19937(seed)."""
        out = np.zeros(n)
        self.lib.ref_uniform(1 if bits64 else 0, seed, lo, hi, n, abi.dptr(out))
        return out

    def _solve(self, kind, grid, b, x, tol, maxit, rep):
        rc = self.lib.ref_poisson_solve(1 if kind == "mg" else 0, C.byref(grid.desc()),
                                        abi.dptr(b), abi.dptr(x), tol, maxit, C.byref(rep))
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def ns(self, grid, cfg):
        return _NS(self.lib, "ref", grid, cfg)

    def load_case(self, path, max_cells=1 << 24):
        """The reference's loadCase (core/src/flow/case.cpp:136-170): grid descriptor, solid
        mask, flow config, run directory and run options (max_steps, snapshot_every,
        checkpoint_every, stop_time, steady_tol)."""
        g, cfg = abi.GridDesc(), abi.FlowConfig()
        solid = np.zeros(max_cells, dtype=np.uint8)
        run_dir = C.create_string_buffer(4096)
        run, runf = (C.c_int * 3)(), np.zeros(2)
        rc = self.lib.ref_load_case(str(path).encode(), C.byref(g), solid.ctypes.data_as(C.POINTER(C.c_uint8)),
                                    max_cells, C.byref(cfg), run_dir, 4096, run, abi.dptr(runf))
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())
        n = g.nx * g.ny * g.nz
        opts = dict(run_dir=run_dir.value.decode(), max_steps=run[0], snapshot_every=run[1],
                    checkpoint_every=run[2], stop_time=float(runf[0]), steady_tol=float(runf[1]))
        return g, solid[:n].copy(), cfg, opts

    def run_case(self, grid, cfg, run_dir, max_steps, stop_time=0.0, steady_tol=0.0, checkpoint_every=0,
                 restart_from=None):
        """The reference's runCase (core/src/flow/case.cpp:349-401): diagnostics.jsonl,
        checkpoints and final.vtu in run_dir. Returns its RunSummary as a dict."""
        out, steady = np.zeros(7), C.c_int()
        rc = self.lib.ref_run_case(C.byref(grid.desc()), C.byref(cfg), str(run_dir).encode(), max_steps,
                                   stop_time, steady_tol, checkpoint_every,
                                   str(restart_from).encode() if restart_from else None, abi.dptr(out),
                                   C.byref(steady))
        if rc:
            raise RuntimeError(self.lib.ref_last_error().decode())
        keys = ("steps", "time", "momentum_residual", "continuity_residual", "mass_error", "cd", "cl")
        d = dict(zip(keys, out.tolist()))
        d["steps"] = int(d["steps"])
        d["steady"] = bool(steady.value)
        return d

    def morton_encode(self, x, y, z):
        return self.lib.ref_morton_encode(x, y, z)

    def octree(self, origin, extent, max_level):
        return RefOctree(self.lib, origin, extent, max_level)


class RefOctree:
    """The reference's nabla::mesh::Octree (core/src/mesh/octree.cpp)."""

    def __init__(self, lib, origin, extent, max_level):
        self.lib = lib
        o = np.asarray(origin, dtype=np.float64)
        e = np.asarray(extent, dtype=np.float64)
        self.h = lib.ref_octree_create(abi.dptr(o), abi.dptr(e), max_level)
        self.max_level = max_level

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_octree_destroy(self.h)
            self.h = None

    def refine_uniform(self, times):
        self.lib.ref_octree_refine_uniform(self.h, times)

    def refine_box(self, lo, hi, times):
        self.lib.ref_octree_refine_box(self.h, abi.dptr(np.asarray(lo, dtype=np.float64)),
                                       abi.dptr(np.asarray(hi, dtype=np.float64)), times)

    def refine_morton(self, key):
        if self.lib.ref_octree_refine_morton(self.h, key):
            raise RuntimeError(self.lib.ref_last_error().decode())

    def coarsen(self, key, level):
        return self.lib.ref_octree_coarsen(self.h, key, level)

    def is_balanced(self):
        return bool(self.lib.ref_octree_is_balanced(self.h))

    def cells(self):
        n = self.lib.ref_octree_cell_count(self.h)
        m = np.zeros(n, dtype=np.uint64)
        lv = np.zeros(n, dtype=np.uint8)
        mk = np.zeros(n, dtype=np.uint8)
        self.lib.ref_octree_cells(self.h, m.ctypes.data_as(C.POINTER(C.c_uint64)),
                                  lv.ctypes.data_as(C.POINTER(C.c_uint8)),
                                  mk.ctypes.data_as(C.POINTER(C.c_uint8)))
        return m, lv, mk

    def set_mask(self, i, mask):
        self.lib.ref_octree_set_mask(self.h, i, mask)

    def center(self, i):
        c = np.zeros(3)
        self.lib.ref_octree_cell_center(self.h, i, abi.dptr(c))
        return c

    def face_neighbors(self, i, d):
        out = (C.c_uint64 * 4)()
        n = self.lib.ref_octree_face_neighbors(self.h, i, d, out)
        return [out[k] for k in range(n)]

    def apply_a(self, x):
        out = np.zeros(len(x))
        self.lib.ref_octree_apply_a(self.h, abi.dptr(np.ascontiguousarray(x, dtype=np.float64)),
                                    abi.dptr(out))
        return out

    def build_diagonal(self):
        n = self.lib.ref_octree_cell_count(self.h)
        d = np.zeros(n)
        self.lib.ref_octree_build_diagonal(self.h, abi.dptr(d))
        return d

    def solve(self, b, tol, maxit):
        x = np.zeros(len(b))
        rep = abi.PoissonReport()
        self.lib.ref_octree_solve(self.h, abi.dptr(np.ascontiguousarray(b, dtype=np.float64)),
                                  abi.dptr(x), tol, maxit, C.byref(rep))
        return x, rep


class _NS:
    """One NSSolver instance in either oracle (same method names as the reference)."""

    def __init__(self, lib, prefix, grid, cfg):
        self.lib, self.p, self.grid = lib, prefix, grid
        self.h = getattr(lib, f"{prefix}_ns_create")(C.byref(grid.desc()), C.byref(cfg))
        if not self.h:
            raise RuntimeError("oracle NS create failed")

    def __del__(self):
        if getattr(self, "h", None):
            getattr(self.lib, f"{self.p}_ns_destroy")(self.h)
            self.h = None

    def initialize(self):
        getattr(self.lib, f"{self.p}_ns_initialize")(self.h)

    def set_state(self, u, v, w, p, step=0, t=0.0, dt_last=0.0):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, p)]
        getattr(self.lib, f"{self.p}_ns_set_state")(self.h, *[abi.dptr(a) for a in arrs], step, t,
                                                      dt_last)

    def get_state(self):
        nu, nv, nw, np_ = self.grid.sizes()
        u, v, w, p = np.zeros(nu), np.zeros(nv), np.zeros(nw), np.zeros(np_)
        getattr(self.lib, f"{self.p}_ns_get_state")(self.h, abi.dptr(u), abi.dptr(v), abi.dptr(w),
                                                      abi.dptr(p))
        return u, v, w, p

    def compute_dt(self):
        return getattr(self.lib, f"{self.p}_ns_compute_dt")(self.h)

    def step(self, dt=0.0):
        rep = abi.StepReport()
        getattr(self.lib, f"{self.p}_ns_step")(self.h, dt, C.byref(rep))
        return rep

    def write_checkpoint(self, path):
        """The reference's writeCheckpoint (core/src/flow/case.cpp:274-294)."""
        if getattr(self.lib, f"{self.p}_ns_write_checkpoint")(self.h, str(path).encode()):
            raise RuntimeError(self.lib.ref_last_error().decode())

    def read_checkpoint(self, path):
        """The reference's readCheckpoint (core/src/flow/case.cpp:296-319)."""
        if getattr(self.lib, f"{self.p}_ns_read_checkpoint")(self.h, str(path).encode()):
            raise RuntimeError(self.lib.ref_last_error().decode())


class Dropin:
    """The reference's own NSSolver / PoissonSolver seams with the B200 library
    plugged in (oracle/_ref/libnabla_dropin.so, built from oracle/dropin_shim.cpp
    and nabla-ai_b200/integration/nabla_flow_cuda.hpp). Modes: 0 the reference's
    CPU MgPoisson, 1 CudaMgPoisson inside the reference NSSolver, 2 CudaNSSolver."""

    def __init__(self, path=DROPIN_PATH):
        L = self.lib = _load(path)
        L.dropin_last_error.restype = C.c_char_p
        L.dropin_run.argtypes = [GP, FP, C.c_int, C.c_int, C.c_double, DP, DP, DP, DP,
                                 C.POINTER(C.c_int), DP]
        L.dropin_poisson.argtypes = [GP, DP, DP, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     DP, C.POINTER(C.c_int)]

    def run(self, grid, cfg, mode, state, nsteps, dt=0.0):
        gd = grid.desc()
        out = [np.array(a, dtype=np.float64, copy=True) for a in state]
        iters = (C.c_int * nsteps)()
        dts = np.zeros(nsteps)
        st = self.lib.dropin_run(C.byref(gd), C.byref(cfg), mode, nsteps, dt,
                                 *[abi.dptr(a) for a in out], iters, abi.dptr(dts))
        if st != 0:
            raise RuntimeError(self.lib.dropin_last_error().decode())
        return out, list(iters), dts

    def backend(self, grid, cfg, nsteps, points):
        """CudaSolverBackend (the SolverBackend seam) against the reference's NSSolver read as
        BaselineBackend reads it: (sample(), sampleMany(), reference) as [4, n] arrays, the
        telemetry (t, dt, cfl, momentum residual, divergence max, poisson iters) of both, and the
        largest difference of sampleFlowCuda from per-cell sample() on a refined reference Octree."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
        n = pts.shape[0]
        one, many, ref, tele, err = np.zeros(4 * n), np.zeros(4 * n), np.zeros(4 * n), np.zeros(12), C.c_double()
        L = self.lib
        L.dropin_backend.argtypes = [GP, FP, C.c_int, C.c_int64, DP, DP, DP, DP, DP, C.POINTER(C.c_double)]
        st = L.dropin_backend(C.byref(grid.desc()), C.byref(cfg), nsteps, n, abi.dptr(pts), abi.dptr(one),
                              abi.dptr(many), abi.dptr(ref), abi.dptr(tele), C.byref(err))
        if st != 0:
            raise RuntimeError(L.dropin_last_error().decode())
        return one.reshape(4, n), many.reshape(4, n), ref.reshape(4, n), tele[:6], tele[6:], err.value

    def poisson(self, grid, b, tol, max_cycles, mode):
        gd = grid.desc()
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        it, res, conv = C.c_int(), C.c_double(), C.c_int()
        st = self.lib.dropin_poisson(C.byref(gd), abi.dptr(b), abi.dptr(x), tol, max_cycles, mode,
                                     C.byref(it), C.byref(res), C.byref(conv))
        if st != 0:
            raise RuntimeError(self.lib.dropin_last_error().decode())
        return x, it.value, res.value, bool(conv.value)
