"""ctypes mirror of include/nabla_b200.h (structs, enums, prototypes).

The shared library is built in-tree by ``nabla-ai_b200/build.py`` into
``nabla-ai_b200/lib/libnabla_b200.so``. Loading fails loudly when it is
missing: there is no Python or CPU fallback for the solver path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libnabla_b200.so")

# status codes (nb_status)
NB_OK = 0
NB_ERR_BAD_ARG = 1
NB_ERR_OOM = 2
NB_ERR_NOT_CONVERGED = 3
NB_ERR_NAN = 4
NB_ERR_DEVICE_TIMEOUT = 5
NB_ERR_CUDA = 6
NB_ERR_UNSUPPORTED = 7

# BoundaryType / InletProfile / ConvectionScheme (core/include/nabla/flow/grid.hpp:17-18)
BC_WALL, BC_INLET, BC_OUTLET, BC_PERIODIC = 0, 1, 2, 3
PROFILE_UNIFORM, PROFILE_PARABOLIC = 0, 1
CONV_CENTRAL, CONV_WENO5 = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1


class FaceBC(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("profile", C.c_int32),
        ("inlet_axis", C.c_int32),
        ("reserved", C.c_int32),
        ("wall_velocity", C.c_double * 3),
        ("inlet_speed", C.c_double),
    ]


class GridDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("reserved", C.c_int32),
        ("origin", C.c_double * 3),
        ("dx", C.c_double),
        ("dy", C.c_double),
        ("dz", C.c_double),
        ("face", FaceBC * 6),
        ("solid", C.POINTER(C.c_uint8)),
    ]


class FlowConfig(C.Structure):
    _fields_ = [
        ("reynolds", C.c_double),
        ("ref_length", C.c_double),
        ("velocity_scale", C.c_double),
        ("density", C.c_double),
        ("cfl", C.c_double),
        ("body_force", C.c_double * 3),
        ("convection", C.c_int32),
        ("poisson_max_iters", C.c_int32),
        ("poisson_tol", C.c_double),
        ("tol_continuity", C.c_double),
        ("tol_mass", C.c_double),
        ("ref_area", C.c_double),
    ]


class StepReport(C.Structure):
    _fields_ = [
        ("step", C.c_int32),
        ("poisson_iters", C.c_int32),
        ("t", C.c_double),
        ("dt", C.c_double),
        ("cfl", C.c_double),
        ("momentum_residual", C.c_double),
        ("continuity_residual", C.c_double),
        ("divergence_max", C.c_double),
        ("mass_error", C.c_double),
        ("poisson_residual", C.c_double),
        ("cd", C.c_double),
        ("cl", C.c_double),
        ("cell_count", C.c_uint64),
        ("accepted", C.c_int32),
        ("converged", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PoissonReport(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("residual", C.c_double)]


class AmrGeom(C.Structure):
    _fields_ = [
        ("nb0", C.c_int32 * 3),
        ("lmax", C.c_int32),
        ("h0", C.c_double * 3),
        ("origin", C.c_double * 3),
        ("face", FaceBC * 6),
    ]


DP = C.POINTER(C.c_double)
VP = C.c_void_p


def dptr(a: np.ndarray | None):
    """Pointer to a contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(DP)


class Tuning(C.Structure):
    """nb_tuning: launch shapes, halo staging, mixed-form sweeps, exact
    coarse-solve threshold and PDL of the objects a context creates."""
    _fields_ = [
        ("mg_ctas_per_sm", C.c_int32),
        ("rhs_ctas_per_sm", C.c_int32),
        ("halo_mode", C.c_int32),
        ("sweeps", C.c_int32),
        ("coarse_direct_max", C.c_int32),
        ("pdl", C.c_int32),
        ("threads_per_brick", C.c_int32),
        ("smoother", C.c_int32),
        ("tail_bricks", C.c_int32),
        ("warm_start", C.c_int32),
        ("vgrid", C.c_int32),
        ("coarse_bf16", C.c_int32),
        ("ghost_map", C.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class TuneReport(C.Structure):
    _fields_ = [
        ("best", Tuning),
        ("best_ms", C.c_double),
        ("default_ms", C.c_double),
        ("candidates", C.c_int32),
        ("rejected", C.c_int32),
        ("from_cache", C.c_int32),
        ("key", C.c_char * 128),
    ]


class RunOptions(C.Structure):
    _fields_ = [("run_dir", C.c_char_p), ("max_steps", C.c_int32), ("checkpoint_every", C.c_int32),
                ("stop_time", C.c_double), ("steady_tol", C.c_double), ("restart_from", C.c_char_p),
                ("precision", C.c_int32), ("snapshot_every", C.c_int32)]


class RunSummary(C.Structure):
    _fields_ = [("steps", C.c_int32), ("steady", C.c_int32), ("time", C.c_double),
                ("momentum_residual", C.c_double), ("continuity_residual", C.c_double),
                ("mass_error", C.c_double), ("cd", C.c_double), ("cl", C.c_double), ("cells", C.c_uint64)]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["steady"] = bool(d["steady"])
        return d


# (name, restype, argtypes) for every symbol declared in include/nabla_b200.h
PROTOTYPES = [
    ("nb_ctx_create", C.c_int, [C.c_int, C.POINTER(VP)]),
    ("nb_ctx_destroy", None, [VP]),
    ("nb_last_error", C.c_char_p, [VP]),
    ("nb_status_string", C.c_char_p, [C.c_int]),
    ("nb_ctx_launch_count", C.c_uint64, [VP]),
    ("nb_ctx_synchronize", C.c_int, [VP]),
    ("nb_ctx_stream", VP, [VP]),
    ("nb_case_create", C.c_int, [VP, C.POINTER(GridDesc), C.POINTER(FlowConfig), C.c_int, C.POINTER(VP)]),
    ("nb_case_destroy", None, [VP]),
    ("nb_case_initialize", C.c_int, [VP]),
    ("nb_case_set_state", C.c_int, [VP, DP, DP, DP, DP, C.c_int, C.c_double, C.c_double]),
    ("nb_case_get_state", C.c_int, [VP, DP, DP, DP, DP]),
    ("nb_case_get_clock", C.c_int, [VP, C.POINTER(C.c_int), DP, DP]),
    ("nb_case_compute_dt", C.c_int, [VP, DP]),
    ("nb_step", C.c_int, [VP, C.c_double, C.POINTER(StepReport)]),
    ("nb_step_many", C.c_int, [VP, C.c_double, C.c_int, C.POINTER(StepReport)]),
    ("nb_batch_step", C.c_int, [VP, C.POINTER(VP), C.c_int, C.c_double, C.c_int, C.POINTER(StepReport)]),
    ("nb_step_async", C.c_int, [VP, C.c_double]),
    ("nb_step_wait", C.c_int, [VP, C.POINTER(StepReport)]),
    ("nb_step_ready", C.c_int, [VP, C.POINTER(C.c_int)]),
    ("nb_case_device_bytes", C.c_uint64, [VP]),
    ("nb_case_cell_count", C.c_uint64, [VP]),
    ("nb_case_stream", VP, [VP]),
    ("nb_ctx_profile", C.c_int, [VP, C.c_char_p]),
    ("nb_case_sample", C.c_int, [VP, C.c_int, C.c_int64, DP, DP]),
    ("nb_amr_case_sensors", C.c_int, [VP, DP]),
    ("nb_amr_case_transfer", C.c_int, [VP, VP]),
    ("nb_amr_coarsen", C.c_int, [C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_uint8),
                                 C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64)]),
    ("nb_case_write_vtu", C.c_int, [VP, C.c_char_p]),
    ("nb_run_case", C.c_int, [VP, C.POINTER(GridDesc), C.POINTER(FlowConfig), C.POINTER(RunOptions),
                              C.POINTER(RunSummary)]),
    ("nb_case_write_checkpoint", C.c_int, [VP, C.c_char_p]),
    ("nb_case_read_checkpoint", C.c_int, [VP, C.c_char_p]),
    ("nb_checkpoint_info", C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int32), DP, DP]),
    ("nb_tuning_default", None, [C.POINTER(Tuning)]),
    ("nb_ctx_set_tuning", C.c_int, [VP, C.POINTER(Tuning)]),
    ("nb_ctx_get_tuning", C.c_int, [VP, C.POINTER(Tuning)]),
    ("nb_autotune", C.c_int, [VP, VP, C.c_int, C.c_char_p, C.POINTER(TuneReport)]),
    ("nb_tune_cache_lookup", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Tuning), DP]),
    ("nb_tune_cache_store", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Tuning), C.c_double]),
    ("nb_ctx_profile_read", C.c_int, [VP, DP, C.POINTER(C.c_uint64), DP]),
    ("nb_poisson_solve", C.c_int, [VP, C.POINTER(GridDesc), DP, DP, C.c_double, C.c_int, C.c_int,
                                   C.POINTER(PoissonReport)]),
    ("nb_apply_laplacian", C.c_int, [VP, C.POINTER(GridDesc), DP, DP]),
    ("nb_apply_laplacian_noalloc", C.c_int, [C.POINTER(GridDesc), VP, VP, VP]),
    ("nb_amr_refine", C.c_int, [C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_uint8),
                                C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64)]),
    ("nb_amr_mesh_create", C.c_int, [VP, C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64,
                                     C.POINTER(C.c_uint8), C.POINTER(VP)]),
    ("nb_amr_mesh_destroy", None, [VP]),
    ("nb_amr_mesh_leaf_count", C.c_int64, [VP]),
    ("nb_amr_mesh_leaves", C.c_int, [VP, C.POINTER(C.c_int32)]),
    ("nb_morton_encode", C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32]),
    ("nb_morton_decode", None, [C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("nb_amr_build_maps", C.c_int, [VP, C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64,
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32)]),
    ("nb_amr_mesh_maps", C.c_int, [VP, C.POINTER(C.c_uint64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("nb_amr_tree_maps", C.c_int, [C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("nb_amr_refine_device", C.c_int, [VP, C.POINTER(AmrGeom), C.POINTER(C.c_int32), C.c_int64,
                                       C.POINTER(C.c_uint8), C.POINTER(C.c_int32), C.c_int64,
                                       C.POINTER(C.c_int64)]),
    ("nb_amr_case_refine", C.c_int, [VP, C.c_int, C.c_double, C.POINTER(C.c_int32), C.c_int64,
                                     C.POINTER(C.c_int64)]),
    ("nb_amr_mesh_couplings", C.c_int, [VP, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        DP, C.c_int64]),
    ("nb_amr_apply_laplacian", C.c_int, [VP, VP, DP, DP]),
    ("nb_amr_poisson_solve", C.c_int, [VP, VP, DP, DP, C.c_double, C.c_int, C.c_int, C.POINTER(PoissonReport)]),
    ("nb_amr_case_create", C.c_int, [VP, VP, C.POINTER(FlowConfig), C.c_int, C.POINTER(VP)]),
    ("nb_amr_case_sizes", C.c_int, [VP, C.POINTER(C.c_int64)]),
    ("nb_amr_case_slabs", C.c_int, [VP, C.c_int, C.POINTER(C.c_int32)]),
    ("nb_amr_case_set_state", C.c_int, [VP, DP, DP, DP, DP]),
    ("nb_amr_case_get_state", C.c_int, [VP, DP, DP, DP, DP]),
]


def declared_symbols() -> list[str]:
    """Function names declared in include/nabla_b200.h (parsed from the header)."""
    import re

    hdr = os.path.join(os.path.dirname(PKG_ROOT), "include", "nabla_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(nb_[a-z0-9_]+)\s*\(", text)))


_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load libnabla_b200.so and attach prototypes. Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python nabla-ai_b200/build.py` "
            "(the CUDA path has no fallback)")
    lib = C.CDLL(p)
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
