"""The multi-rank plumbing of bench.py --gpus N (independent replicas), run
as two gloo ranks on the CPU: the maximum of per-rank times, the barrier and
the whole-job throughput."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from carpet_b200 import replicas
    replicas.init("gloo", timeout_s=30)
    assert replicas.world() == (world, rank) and replicas.active()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
    replicas.barrier()
    m = replicas.max_over_ranks(ms, device="cpu")
    out.put((rank, m, replicas.job_throughput(1e9, world, m)))
    replicas.finish()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    for _, m, thr in res:
        assert m == 15.0
        assert thr == pytest.approx(2e9 / 15e-3)


def test_single_process_is_its_own_maximum():
    from carpet_b200 import replicas
    assert not replicas.active()
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_throughput(100.0, 1, 10.0) == pytest.approx(1e4)
