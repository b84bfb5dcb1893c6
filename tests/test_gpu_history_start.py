"""History warm starts of the mixed form (nb_tuning.warm_start = 2 or 3):
after two steps of history each projection's MG-PCG starts from the same RK
stage's pressure extrapolated linearly in time over the last two steps (2),
or from that stage's pressure one step ago corrected by how the previous
stage's pressure has changed since, scaled to this stage (3); both scaled by
this step's dt. Before two steps of history, the scaled last pressure. The solve
still stops on ||r|| <= tol ||b|| (and the true residual), so the state stays
within the mixed form's bar of the FP64 form while the cycles drop. A new
state clears the history: stepping from set_state repeats the run."""
import numpy as np
import pytest

from helpers import rel_err
from nabla_b200 import abi, solver
from test_gpu_tuning import _channel

pytestmark = pytest.mark.gpu


def _run(ctx, tuning, precision=abi.PRECISION_MIXED, nsteps=8):
    ctx.set_tuning(**tuning)
    try:
        ac = _channel(ctx, precision)
        cycles = []
        for _ in range(nsteps):
            rep = ac.step(0.004)
            assert rep.converged and rep.divergence_max <= 1e-8
            cycles.append(rep.poisson_iters)
        return ac, ac.get_state(), cycles
    finally:
        ctx.set_tuning(**solver.default_tuning())


@pytest.mark.parametrize("mode", [2, 3])
def test_history_start_tracks_fp64_with_fewer_cycles(ctx, mode):
    _, ref, _ = _run(ctx, {}, abi.PRECISION_FP64)
    _, scaled, c1 = _run(ctx, dict(warm_start=1))
    _, hist, c2 = _run(ctx, dict(warm_start=mode))
    for a in range(3):
        assert rel_err(hist[a], ref[a]) <= 1e-6
    assert c2[:2] == c1[:2]  # no history yet: the scaled start
    print(f"cycles per step, scaled start: {c1}, history start {mode}: {c2}")
    assert sum(c2[2:]) < sum(c1[2:])


def test_new_state_clears_history(ctx):
    """A state that differs from the resident one clears the history, so stepping
    from it repeats exactly."""
    ac, st, _ = _run(ctx, {}, nsteps=3)
    first = [np.array(a, copy=True) for a in st]
    for _ in range(2):
        ac.step(0.004)
    ac.set_state(*first)  # differs from the resident state: history cleared
    a = [ac.step(0.004).poisson_iters for _ in range(4)]
    sa = [np.array(x, copy=True) for x in ac.get_state()]
    ac.set_state(*first)
    b = [ac.step(0.004).poisson_iters for _ in range(4)]
    assert a == b and a[:2] != [0, 0]
    for x, y in zip(sa, ac.get_state()):
        assert np.array_equal(x, y)


def test_round_trip_upload_keeps_history(ctx):
    """Reading the state back and uploading it unchanged every step (a host round
    trip) keeps the history: the same cycles and bits as stepping on the device."""
    a, _, ca = _run(ctx, {}, nsteps=6)
    ctx.set_tuning(**solver.default_tuning())
    b = _channel(ctx, abi.PRECISION_MIXED)
    cb = []
    for _ in range(6):
        st = [np.array(x, copy=True) for x in b.get_state()]
        b.set_state(*st)
        cb.append(b.step(0.004).poisson_iters)
    assert cb == ca
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
