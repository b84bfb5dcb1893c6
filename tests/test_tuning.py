"""Launch tuning on the host: the default nb_tuning and the tuning cache file
(nb_tune_cache_lookup / nb_tune_cache_store). No GPU is needed."""
import ctypes as C

import pytest

from nabla_b200 import abi, solver


def _lib():
    return abi.load()


def test_default_tuning():
    assert solver.default_tuning() == {"mg_ctas_per_sm": 4, "rhs_ctas_per_sm": 4, "halo_mode": 0, "sweeps": 2,
                                       "coarse_direct_max": 256, "pdl": 1, "threads_per_brick": 512,
                                       "smoother": 1, "tail_bricks": 8, "warm_start": 3,
                                       "vgrid": 0, "coarse_bf16": 0, "ghost_map": 1}


def _tuning(**kw):
    t = abi.Tuning()
    _lib().nb_tuning_default(C.byref(t))
    for k, v in kw.items():
        setattr(t, k, v)
    return t


def test_cache_round_trip(tmp_path):
    lib = _lib()
    path = str(tmp_path / "tune.txt").encode()
    out = abi.Tuning()
    ms = C.c_double()
    assert lib.nb_tune_cache_lookup(path, b"gpu/a", C.byref(out), C.byref(ms)) == 0  # no file yet
    assert lib.nb_tune_cache_store(path, b"gpu/a", C.byref(_tuning(sweeps=1, pdl=0)), 1.5) == abi.NB_OK
    assert lib.nb_tune_cache_store(path, b"gpu/b", C.byref(_tuning(mg_ctas_per_sm=2)), 2.5) == abi.NB_OK
    assert lib.nb_tune_cache_lookup(path, b"gpu/a", C.byref(out), C.byref(ms)) == 1
    assert out.sweeps == 1 and out.pdl == 0 and ms.value == 1.5
    # a store replaces the key's line and keeps the others
    assert lib.nb_tune_cache_store(path, b"gpu/a", C.byref(_tuning(halo_mode=1)), 0.75) == abi.NB_OK
    assert lib.nb_tune_cache_lookup(path, b"gpu/a", C.byref(out), C.byref(ms)) == 1
    assert out.halo_mode == 1 and out.sweeps == 2 and ms.value == 0.75
    assert lib.nb_tune_cache_lookup(path, b"gpu/b", C.byref(out), C.byref(ms)) == 1
    assert out.mg_ctas_per_sm == 2
    text = (tmp_path / "tune.txt").read_text().splitlines()
    assert len(text) == 2
    assert lib.nb_tune_cache_lookup(path, b"gpu/c", C.byref(out), C.byref(ms)) == 0


@pytest.mark.parametrize("field,value", [("mg_ctas_per_sm", 0), ("mg_ctas_per_sm", 17), ("rhs_ctas_per_sm", 5),
                                         ("halo_mode", 2), ("sweeps", 4), ("coarse_direct_max", 513), ("pdl", 2),
                                         ("threads_per_brick", 64), ("threads_per_brick", 384),
                                         ("smoother", 2), ("tail_bricks", -1), ("tail_bricks", 4097),
                                         ("warm_start", 4), ("vgrid", 2), ("coarse_bf16", 2),
                                         ("ghost_map", 2)])
def test_cache_rejects_out_of_range_tuning(tmp_path, field, value):
    path = str(tmp_path / "tune.txt").encode()
    assert _lib().nb_tune_cache_store(path, b"k", C.byref(_tuning(**{field: value})), 1.0) == abi.NB_ERR_BAD_ARG


def test_cache_rejects_bad_key_and_malformed_file(tmp_path):
    lib = _lib()
    path = tmp_path / "tune.txt"
    assert lib.nb_tune_cache_store(str(path).encode(), b"a key", C.byref(_tuning()), 1.0) == abi.NB_ERR_BAD_ARG
    path.write_text("# comment\n\ngpu/a 4 4 0 2 256 1 512 1 8 0 0 0 1 1.0\ngpu/b 4 2\n")
    out = abi.Tuning()
    assert lib.nb_tune_cache_lookup(str(path).encode(), b"gpu/a", C.byref(out), None) == 1
    assert lib.nb_tune_cache_lookup(str(path).encode(), b"gpu/b", C.byref(out), None) == -1
