"""Multi-GPU runs are replicas only: every rank steps its own cases with no
data-path collective, and the bench reduces only its timings (max over
ranks) before rank 0 prints the whole-job throughput. The reduction runs
here as two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    sys.path.insert(0, REPO)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # each rank's own device time for K steps (ms); rank 1 is the slower
        elapsed = 100.0 + 50.0 * rank
        emax = bench.max_over_ranks(elapsed, world, "cpu")
        cells, steps = 260096, 5
        value = world * cells * steps / (emax * 1e-3) / 1e6
        out.put((rank, emax, value))
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [150.0, 150.0]  # every rank sees the slowest rank's time
    expect = 2 * 260096 * 5 / 0.150 / 1e6  # all ranks' cell-steps over that time
    assert all(abs(r[2] - expect) < 1e-9 * expect for r in res)
