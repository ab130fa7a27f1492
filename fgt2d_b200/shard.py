"""Spatial shard of one transform over several GPUs, one rank per GPU.

The C library partitions the cut-level boxes into Morton ranges of nearly
equal point counts (every rank computes the same partition from the same
replicated points) and keeps, on each rank, the tasks of the boxes it owns
(``fgt_plan_create_shard``, include/fgt_b200.h).  The transform then runs in
two phases with one exchange between them: after phase 1 (formation and
merge) each rank sends the cut-level multipole expansions that another
rank's mp -> loc tasks read across the range boundary (the coupling of
2d/planewave/src/fgt2d.f:1026-1064, 3d/planewave/src/fgt3d.f:1172-1209) and
receives the ones its own tasks read; phase 2 runs mp -> loc, split,
evaluation, the near field and the scatter.  The sum of the ranks' outputs
is the one-GPU result bit for bit.

``exchange`` is the transfer itself over torch.distributed point-to-point
operations (NCCL between GPUs; gloo for the CPU tests), written against
pack / unpack callables so the same code moves device buffers of a plan or
host arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import FGTError, _check, _f64, _p, lib

_ll = ctypes.c_longlong


def exchange(world: int, rank: int, counts, slot_len: int, pack, unpack, device, dtype=None):
    """One exchange of cut-level expansions with every peer.

    counts(peer) -> (nsend, nrecv) in expansions; pack(peer, buf) fills a
    send buffer of nsend * slot_len values; unpack(peer, buf) consumes a
    receive buffer.  All sends and receives are posted together
    (batch_isend_irecv), so the order of peers cannot deadlock; ranks that
    exchange nothing take part in no operation."""
    import torch
    import torch.distributed as dist
    dtype = dtype or torch.float64
    ops, recv = [], []
    for peer in range(world):
        if peer == rank:
            continue
        ns, nr = counts(peer)
        if ns > 0:
            buf = torch.empty(int(ns) * slot_len, dtype=dtype, device=device)
            pack(peer, buf)
            ops.append(dist.P2POp(dist.isend, buf, peer))
        if nr > 0:
            buf = torch.empty(int(nr) * slot_len, dtype=dtype, device=device)
            recv.append((peer, buf))
            ops.append(dist.P2POp(dist.irecv, buf, peer))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for peer, buf in recv:
        unpack(peer, buf)


class HostShard:
    """Host-only view of one rank's shard (no GPU): exchange lists as mp slot
    numbers and task statistics of the filtered plan."""

    def __init__(self, dim, nd, delta, eps, sources, targ, ifpgh, ifpghtarg, nranks, rank):
        L = lib()
        src = _f64(sources, (-1, dim))
        trg = _f64(targ, (-1, dim)) if targ is not None else None
        self.nranks, self.rank = nranks, rank
        h = ctypes.c_void_p()
        _check(L.fgt_host_shard_create(dim, nd, delta, eps, src.shape[0], _p(src),
                                       0 if trg is None else trg.shape[0], _p(trg), ifpgh, ifpghtarg,
                                       nranks, rank, ctypes.byref(h)), "fgt_host_shard_create")
        self._h = h

    def counts(self, peer):
        a, b = _ll(), _ll()
        _check(lib().fgt_host_shard_counts(self._h, peer, ctypes.byref(a), ctypes.byref(b)),
               "fgt_host_shard_counts")
        return a.value, b.value

    def slots(self, peer, which):
        n = self.counts(peer)[0 if which == "send" else 1]
        out = np.zeros(max(n, 1), dtype=np.int32)
        _check(lib().fgt_host_shard_slots(self._h, peer, 0 if which == "send" else 1,
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "fgt_host_shard_slots")
        return out[:n]

    def stats(self):
        o = np.zeros(8, dtype=np.int64)
        _check(lib().fgt_host_shard_stats(self._h, o.ctypes.data_as(ctypes.POINTER(_ll))),
               "fgt_host_shard_stats")
        keys = ["owned_sources", "owned_targets", "form_tasks", "eval_tasks", "direct_tasks",
                "m2l_tasks", "shift_tasks", "mp_slots"]
        return {k: int(v) for k, v in zip(keys, o)}

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_host_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ShardPlan:
    """One rank's plan of a sharded transform (charges, potentials)."""

    def __init__(self, ctx, dim, nd, delta, eps, sources, targ, ifpgh, ifpghtarg, nranks, rank):
        L = lib()
        src = _f64(sources, (-1, dim))
        trg = _f64(targ, (-1, dim)) if targ is not None else None
        self.ctx, self.nd, self.nranks, self.rank = ctx, nd, nranks, rank
        self.ns, self.nt = src.shape[0], 0 if trg is None else trg.shape[0]
        h = ctypes.c_void_p()
        _check(L.fgt_plan_create_shard(ctx.handle, dim, nd, delta, eps, self.ns, _p(src), self.nt, _p(trg),
                                       ifpgh, ifpghtarg, nranks, rank, ctypes.byref(h)),
               "fgt_plan_create_shard")
        self._h = h

    def counts(self, peer):
        a, b, c = _ll(), _ll(), _ll()
        _check(lib().fgt_plan_shard_counts(self._h, peer, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "fgt_plan_shard_counts")
        return a.value, b.value

    def slot_doubles(self):
        a, b, c = _ll(), _ll(), _ll()
        _check(lib().fgt_plan_shard_counts(self._h, 0, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "fgt_plan_shard_counts")
        return c.value

    def owned(self):
        a, b = _ll(), _ll()
        _check(lib().fgt_plan_shard_owned(self._h, ctypes.byref(a), ctypes.byref(b)), "fgt_plan_shard_owned")
        return a.value, b.value

    def phase(self, p, d_chg, d_pot, d_pt, stream=None):
        _check(lib().fgt_plan_execute_device_phase(self._h, p, d_chg, d_pot or None, d_pt or None, stream),
               "fgt_plan_execute_device_phase")

    def pack(self, peer, d_buf, stream=None):
        _check(lib().fgt_plan_mp_pack(self._h, peer, d_buf, stream), "fgt_plan_mp_pack")

    def unpack(self, peer, d_buf, stream=None):
        _check(lib().fgt_plan_mp_unpack(self._h, peer, d_buf, stream), "fgt_plan_mp_unpack")

    def execute(self, d_chg, d_pot, d_pt, stream=None):
        """Phase 1, the exchange with every peer over torch.distributed
        (device buffers on this rank's GPU), phase 2."""
        import torch
        self.phase(1, d_chg, d_pot, d_pt, stream)
        if self.nranks > 1:
            torch.cuda.current_stream().synchronize() if stream is None else torch.cuda.synchronize()
            dev = torch.device("cuda", torch.cuda.current_device())
            exchange(self.nranks, self.rank, self.counts, self.slot_doubles(),
                     lambda peer, buf: (self.pack(peer, buf.data_ptr(), stream), torch.cuda.synchronize()),
                     lambda peer, buf: self.unpack(peer, buf.data_ptr(), stream), dev)
            torch.cuda.synchronize()
        self.phase(2, d_chg, d_pot, d_pt, stream)

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["exchange", "HostShard", "ShardPlan", "FGTError"]
