"""MBIR of one volume split across ranks by slices (slab sharding).

The reference's multi-GPU scheme (``src/dist_array.h:349-373``,
``src/multiproc.h:95-118``, ``src/tv_update.cpp:82-96``): every slice is
independent except for the 3-D qGGMRF prior, so each rank owns a slab of
slices and, per attempt of ``Optimizer::run2``,

* exchanges one halo plane with each neighbour for the buffers the attempt
  reads (x and sol, or one buffer when they coincide); at an end of the
  volume the halo is a copy of the slab's own edge plane, which reproduces
  the clamp-to-edge stencil;
* runs the attempt on its slab (``tc_slab_attempt``): the fused update, H new
  and six FP64 sums of the step test;
* sums the six values over all ranks and applies the step test
  (``tc_slab_decide``), identically everywhere.

``solve_slab`` runs one rank's slab with an exchanger; ``TorchExchange`` does
the exchange and the sum with ``torch.distributed`` (NCCL point-to-point
transfers and an all-reduce, one process per GPU).  ``solve_slabs_local``
runs several slabs of one process in lockstep (the exchange is a device
copy), which checks the sharded algorithm against the whole-volume solve on
one GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .plan import Plan, _check_tensor, _ptr, _stream


class _DevView:
    """A device array as a torch tensor without a copy (CUDA array interface)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _view(ptr: int, n: int, typestr: str = "<f4"):
    import torch
    return torch.as_tensor(_DevView(ptr, n, typestr), device="cuda")


class Slab:
    """One rank's slab: ``aty`` and ``x0`` are its owned slices [S][n][n]
    (CUDA float32), ``sino_sq`` the whole volume's ||y||^2."""

    def __init__(self, plan: Plan, aty, sino_sq: float, x0, num_iters: int, sigma: float,
                 p: float = 1.2, prior_weight: float = 1.0, step: float = 0.0, max_attempts: int = 0):
        S = x0.shape[0]
        _check_tensor(aty, (S, plan.n, plan.n), "aty")
        _check_tensor(x0, (S, plan.n, plan.n), "x0")
        self.plan, self.S, self.K, self.n = plan, S, int(num_iters), plan.n
        o = _lib.MbirOpts()
        _lib.lib().tc_mbir_opts_default(ctypes.byref(o))
        o.num_iters, o.sigma, o.p, o.prior_weight = self.K, float(sigma), float(p), float(prior_weight)
        o.step, o.use_graph, o.max_attempts = float(step), 0, int(max_attempts)
        h = ctypes.c_void_p()
        _lib.call("tc_slab_create", plan._h, _ptr(aty), float(sino_sq), _ptr(x0), S, ctypes.byref(o),
                  ctypes.byref(h), _stream())
        self._h = h
        self.cond = self.K > 0

    def halo(self, which: int):
        """(send_lo, send_hi, recv_lo, recv_hi, same) for x (0) or sol (1)."""
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        same = ctypes.c_int()
        _lib.call("tc_slab_halo", self._h, int(which), *[ctypes.byref(q) for q in ptrs], ctypes.byref(same))
        plane = self.n * self.n
        return tuple(_view(q.value, plane) for q in ptrs) + (bool(same.value),)

    def attempt(self):
        """Runs one attempt; returns the six local sums (a device view)."""
        q = ctypes.c_void_p()
        _lib.call("tc_slab_attempt", self._h, ctypes.byref(q), _stream())
        return _view(q.value, 6, "<f8")

    def decide(self) -> bool:
        c = ctypes.c_int()
        _lib.call("tc_slab_decide", self._h, ctypes.byref(c), _stream())
        self.cond = bool(c.value)
        return self.cond

    def result(self):
        """(x [S][n][n], history [num_iters][3])."""
        import torch
        x = torch.empty((self.S, self.n, self.n), dtype=torch.float32, device="cuda")
        hist = np.zeros((max(self.K, 1), 3), dtype=np.float64)
        it = ctypes.c_int()
        _lib.call("tc_slab_result", self._h, _ptr(x), hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                  ctypes.byref(it), _stream())
        return x, hist[:self.K]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().tc_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TorchExchange:
    """Halo exchange and sum over ``torch.distributed`` ranks (one slab per
    rank, ranks ordered by slices).  ``halo`` sends the lower boundary plane to
    rank - 1 and the upper one to rank + 1 and receives their planes into the
    halo planes; at an end of the volume the halo is a copy of the own edge
    plane.  ``allreduce`` sums in place."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def halo(self, send_lo, send_hi, recv_lo, recv_hi):
        dist = self.dist
        ops = []
        if self.rank > 0:
            ops.append(dist.P2POp(dist.isend, send_lo, self._peer(self.rank - 1), self.group))
            ops.append(dist.P2POp(dist.irecv, recv_lo, self._peer(self.rank - 1), self.group))
        else:
            recv_lo.copy_(send_lo)
        if self.rank < self.world - 1:
            ops.append(dist.P2POp(dist.isend, send_hi, self._peer(self.rank + 1), self.group))
            ops.append(dist.P2POp(dist.irecv, recv_hi, self._peer(self.rank + 1), self.group))
        else:
            recv_hi.copy_(send_hi)
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def allreduce(self, sums):
        self.dist.all_reduce(sums, group=self.group)

    def _peer(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)


def _exchange_halos(slab: Slab, ex):
    send_lo, send_hi, recv_lo, recv_hi, same = slab.halo(0)
    ex.halo(send_lo, send_hi, recv_lo, recv_hi)
    if not same:
        send_lo, send_hi, recv_lo, recv_hi, _ = slab.halo(1)
        ex.halo(send_lo, send_hi, recv_lo, recv_hi)


def solve_slab(slab: Slab, ex):
    """Runs this rank's slab to the end; every rank calls it with its own slab
    and exchanger.  Returns (x, history) of the slab."""
    while slab.cond:
        _exchange_halos(slab, ex)
        sums = slab.attempt()
        ex.allreduce(sums)
        slab.decide()
    return slab.result()


def solve_slabs_local(slabs):
    """Runs the slabs of one process (consecutive slabs of one volume, one
    GPU) in lockstep: the halo exchange is a device copy between the slabs'
    planes and the sum is taken over the slabs.  Returns [(x, history)]."""
    import torch
    slabs = list(slabs)
    while slabs[0].cond:
        for which in (0, 1):
            views = [s.halo(which) for s in slabs]
            if which == 1 and all(v[4] for v in views):
                break
            for k, (send_lo, send_hi, recv_lo, recv_hi, _) in enumerate(views):
                recv_lo.copy_(views[k - 1][1] if k > 0 else send_lo)
                recv_hi.copy_(views[k + 1][0] if k + 1 < len(slabs) else send_hi)
        sums = [s.attempt() for s in slabs]
        total = torch.stack(sums).sum(0)
        for s in sums:
            s.copy_(total)
        conds = [s.decide() for s in slabs]
        if len(set(conds)) != 1:
            raise RuntimeError("slabs disagree on the step test")
    return [s.result() for s in slabs]
