"""Multi-rank replica plumbing (the bench's N > 1 path) on CPU with gloo,
world size 2: barrier, max over ranks and the whole-job rate."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from tomocam_b200.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    assert (r.rank, r.world) == (rank, world)
    r.barrier()
    # per-rank elapsed times; the slowest rank sets the job's time
    t = 1.0 + rank
    tmax = r.max_over_ranks(t)
    rate = r.aggregate_rate(256 * 20, tmax)
    r.barrier()
    out.put((rank, tmax, rate))
    r.close()


@pytest.mark.timeout(120)
def test_two_rank_replicas_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    for _, tmax, rate in res:
        assert tmax == 2.0                      # max over ranks, seen by every rank
        assert rate == pytest.approx(2 * 256 * 20 / 2.0)   # all ranks' units / slowest time


def test_single_rank_is_a_no_op(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    from tomocam_b200.replicas import Replicas
    r = Replicas("gloo")
    assert r.world == 1 and r.max_over_ranks(3.5) == 3.5
    r.barrier()
    assert r.aggregate_rate(100, 2.0) == 50.0
    r.close()
