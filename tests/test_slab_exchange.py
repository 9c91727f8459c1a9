"""Slab sharding plumbing on CPU with gloo, world size 3: the halo exchange
of tomocam_b200.slab.TorchExchange (neighbours' boundary planes, copies of
the own edge plane at the ends of the volume), the sum of the step-test
values, and the per-rank driver solve_slab with a stand-in slab."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _FakeSlab:
    """Stands in for tomocam_b200.slab.Slab on CPU: two buffers (x, sol)
    with halo planes; an attempt checks that the halos hold what the
    neighbours sent and returns sums that the driver adds over the ranks."""

    def __init__(self, rank, world, plane=5, attempts=4):
        import torch
        self.rank, self.world, self.left = rank, world, attempts
        self.buf = [torch.zeros(4, plane), torch.zeros(4, plane)]   # [halo, owned, owned, halo]
        for b, base in ((0, 100), (1, 200)):
            self.buf[b][1] = base + 10 * rank + 1
            self.buf[b][2] = base + 10 * rank + 2
        self.same = False
        self.cond = True
        self.seen = []

    def halo(self, which):
        b = self.buf[which]
        return b[1], b[2], b[0], b[3], self.same

    def attempt(self):
        import torch
        for which, base in ((0, 100), (1, 200)):
            if which == 1 and self.same:
                continue                     # one buffer: only x was exchanged
            b = self.buf[which]
            lo = base + 10 * (self.rank - 1) + 2 if self.rank > 0 else base + 10 * self.rank + 1
            hi = base + 10 * (self.rank + 1) + 1 if self.rank < self.world - 1 else base + 10 * self.rank + 2
            assert float(b[0, 0]) == lo and float(b[3, 0]) == hi
            b[0].zero_()
            b[3].zero_()
        return torch.full((6,), float(self.rank + 1), dtype=torch.float64)

    def decide_with(self, sums):
        self.seen.append(float(sums[0]))
        self.left -= 1
        self.same = self.left % 2 == 0          # alternate one / two exchanged buffers
        self.cond = self.left > 0
        return self.cond


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    from tomocam_b200.slab import TorchExchange, solve_slab
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ex = TorchExchange()
    # one exchange: the halos get the neighbours' planes or the own edge plane
    send_lo, send_hi = torch.full((3,), 10.0 * rank + 1), torch.full((3,), 10.0 * rank + 2)
    recv_lo, recv_hi = torch.zeros(3), torch.zeros(3)
    ex.halo(send_lo, send_hi, recv_lo, recv_hi)
    sums = torch.full((6,), float(rank + 1), dtype=torch.float64)
    ex.allreduce(sums)
    # the driver loop with a stand-in slab
    fake = _FakeSlab(rank, world)

    class _Drive:
        cond = True

        def halo(self, which):
            return fake.halo(which)

        def attempt(self):
            return fake.attempt()

        def decide(self):
            self.cond = fake.decide_with(self._sums)
            return self.cond

        def result(self):
            return None, fake.seen

    d = _Drive()

    class _Ex:
        def halo(self, *a):
            ex.halo(*a)

        def allreduce(self, s):
            ex.allreduce(s)
            d._sums = s

    _, seen = solve_slab(d, _Ex())
    dist.barrier()
    out.put((rank, float(recv_lo[0]), float(recv_hi[0]), float(sums[0]), seen))
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_three_rank_halo_exchange_and_sum_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 3
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, lo, hi, s, seen in res:
        assert lo == (10.0 * (rank - 1) + 2 if rank > 0 else 10.0 * rank + 1)
        assert hi == (10.0 * (rank + 1) + 1 if rank < world - 1 else 10.0 * rank + 2)
        assert s == 6.0                          # 1 + 2 + 3
        assert seen == [6.0] * 4                 # four attempts, sums over all ranks
