"""Halo exchange between processes that each advance some of the blocks: the
reference's multi-process path (ParallelFace, Mesh.h:62-102; the MPI set-up
of Driver.cu:80-82, 252-254), which it leaves unfinished.

Every process holds the whole arena (all blocks, the layout of
cc_block_arena) and advances its own blocks.  The halo program is the same
on every process; what a process's own blocks' halo is computed from
(cc_halo_dependencies) may lie in blocks other processes own.  Before the
halo program of a stage, each process therefore receives those points from
their owners and sends the points of its own blocks that the others read.
After the exchange every source of a process's own halo holds its owner's
value, so the halo of its blocks equals the single-process one.

Sources are points of the current state (which 0) or of the previous one
(which 1: ghosts no face writes carry their previous value forward).  The
transport is torch.distributed point-to-point messages of the packed values,
one message per peer and state (gloo for host arrays, NCCL for device
arrays); every process computes the whole plan from the same mesh, so the
sizes of all messages are known on both sides and no sizes are exchanged.

DistributedStep runs it inside cc_step: the library calls its hook between
each stage's kernels (which advance only this process's blocks,
cc_set_owned_blocks) and the stage's halo program, and on the local next
time step, which becomes the minimum over processes; the residual's sums are
added over processes.
"""
import ctypes

import numpy as np


def partition(sizes, n_ranks):
    """Owner rank of each block: largest blocks first, each to the rank with
    the fewest points so far (ties to the lower rank)."""
    load = [0] * n_ranks
    owner = [0] * len(sizes)
    for b in sorted(range(len(sizes)), key=lambda b: (-sizes[b], b)):
        r = min(range(n_ranks), key=lambda r: (load[r], r))
        owner[b] = r
        load[r] += sizes[b]
    return owner


class ExchangePlan:
    """The points each process sends to and receives from every other one.

    send[q][w] / recv[q][w]: sorted arena indices of state w (0 current,
    1 previous) that this rank sends to / receives from rank q."""

    def __init__(self, driver, owner, rank, n_ranks):
        if len(owner) != len(driver.field):
            raise ValueError("one owner per block")
        self.rank, self.n_ranks = rank, n_ranks
        dst, src, which = driver.halo_dependencies()
        spans = np.array([driver.block_arena(b) for b in range(len(owner))], dtype=np.int64).reshape(-1, 2)
        first = spans[:, 0]
        owner = np.asarray(owner, dtype=np.int64)

        def owner_of(idx):
            b = np.searchsorted(first, idx, side="right") - 1
            inside = (b >= 0) & (idx < first[np.maximum(b, 0)] + spans[np.maximum(b, 0), 1])
            if not inside.all():
                raise ValueError("a halo dependency lies outside every block")
            return owner[b]

        reader, holder = owner_of(dst), owner_of(src)
        cross = reader != holder
        reader, holder, src, which = reader[cross], holder[cross], src[cross], which[cross]
        self.send = {q: {} for q in range(n_ranks) if q != rank}
        self.recv = {q: {} for q in range(n_ranks) if q != rank}
        for w in (0, 1):
            for q in range(n_ranks):
                if q == rank:
                    continue
                sel_out = (holder == rank) & (reader == q) & (which == w)
                sel_in = (holder == q) & (reader == rank) & (which == w)
                self.send[q][w] = np.unique(src[sel_out])
                self.recv[q][w] = np.unique(src[sel_in])

    def volume(self):
        """Points this rank sends and receives per exchange."""
        out = sum(len(v) for d in self.send.values() for v in d.values())
        inn = sum(len(v) for d in self.recv.values() for v in d.values())
        return out, inn

    def exchange(self, states, group=None):
        """Exchange in place.  states[w] is a list of torch tensors, one per
        field, each indexed by arena point (shape [..., N] flattened to the
        last axis), for state w = 0 (current) and 1 (previous); every field of
        a state is packed into one message per peer."""
        import torch
        import torch.distributed as dist

        for fields in states:
            for f in fields:
                if not f.is_contiguous():
                    raise ValueError("exchange needs contiguous field tensors (it writes through a flat view)")
        reqs, landing = [], []
        for q in sorted(self.send):
            for w in (0, 1):
                fields = states[w]
                idx_out, idx_in = self.send[q][w], self.recv[q][w]
                if len(idx_out):
                    i = torch.as_tensor(idx_out, device=fields[0].device)
                    buf = torch.stack([f.reshape(-1).index_select(0, i) for f in fields])
                    reqs.append(dist.isend(buf.contiguous(), dst=q, group=group, tag=w))
                if len(idx_in):
                    buf = torch.empty((len(fields), len(idx_in)), dtype=fields[0].dtype, device=fields[0].device)
                    reqs.append(dist.irecv(buf, src=q, group=group, tag=w))
                    landing.append((fields, idx_in, buf))
        for r in reqs:
            r.wait()
        for fields, idx_in, buf in landing:
            i = torch.as_tensor(idx_in, device=fields[0].device)
            for f, row in zip(fields, buf):
                f.reshape(-1).index_copy_(0, i, row)


class DistributedStep:
    """Multi-process stepping of one Driver: this process advances the blocks
    `owner` gives it; before every stage's halo program the points its halo
    reads from other processes' blocks arrive through ExchangePlan (packed on
    the device as FP64 rows of every field, sent over torch.distributed), and
    the next time step and the residual are reduced over processes in FP64.
    Construct it before initialize_computation, on a driver that holds the
    whole initial state (every block): the initial time step is reduced over
    processes through the same hook, so every process initialises together."""

    def __init__(self, driver, owner, rank, n_ranks, group=None):
        from . import EXCHANGE_FN, _check

        self.driver, self.rank, self.n_ranks, self.group = driver, rank, n_ranks, group
        self.plan = ExchangePlan(driver, owner, rank, n_ranks)
        lib, ctx = driver.lib, driver.ctx
        mine = np.array([b for b, o in enumerate(owner) if o == rank], dtype=np.int32)
        _check(lib.cc_set_owned_blocks(ctx, mine.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(mine)))
        nf = ctypes.c_int()
        _check(lib.cc_exchange_fields(ctx, ctypes.byref(nf)))
        self.n_fields = nf.value
        self.error = None
        self._hook = EXCHANGE_FN(self._on_event)  # kept alive with self
        _check(lib.cc_set_exchange(ctx, ctypes.cast(self._hook, ctypes.c_void_p), None))

    def _transfer(self):
        import torch
        import torch.distributed as dist
        from . import _check

        lib, ctx = self.driver.lib, self.driver.ctx
        reqs, landing = [], []
        for q in sorted(self.plan.send):
            for w in (0, 1):
                out_idx, in_idx = self.plan.send[q][w], self.plan.recv[q][w]
                if len(out_idx):
                    idx = np.ascontiguousarray(out_idx, dtype=np.int64)
                    buf = np.empty((self.n_fields, len(idx)))
                    _check(lib.cc_pack_points(ctx, w, idx.ctypes.data_as(ctypes.c_void_p), len(idx),
                                              buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
                    reqs.append(dist.isend(torch.from_numpy(buf), dst=q, group=self.group, tag=w))
                if len(in_idx):
                    buf = torch.empty((self.n_fields, len(in_idx)), dtype=torch.float64)
                    reqs.append(dist.irecv(buf, src=q, group=self.group, tag=w))
                    landing.append((w, np.ascontiguousarray(in_idx, dtype=np.int64), buf))
        for r in reqs:
            r.wait()
        for w, idx, buf in landing:
            vals = np.ascontiguousarray(buf.numpy())
            _check(lib.cc_unpack_points(ctx, w, idx.ctypes.data_as(ctypes.c_void_p), len(idx),
                                        vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def _on_event(self, user, event, stage, value):
        from . import CC_EXCHANGE_STAGE

        try:
            if event == CC_EXCHANGE_STAGE:
                self._transfer()
            else:
                import torch
                import torch.distributed as dist

                t = torch.tensor([value[0]], dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
                value[0] = float(t.item())
            return 0
        except Exception as e:  # reported by cc_step as a failed hook
            self.error = e
            return 1

    def residual(self):
        """Driver::compute_residual over every process's points: the sums of
        squared changes and the point counts added over processes, FP64."""
        import torch
        import torch.distributed as dist
        from . import _check

        sums, cnt = np.zeros(4), ctypes.c_int64()
        _check(self.driver.lib.cc_residual_sums(self.driver.ctx, sums.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                ctypes.byref(cnt)))
        t = torch.tensor(list(sums) + [float(cnt.value)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        v = t.numpy()
        return np.sqrt(v[:4] / v[4])

    def close(self):
        """Removes the hook (before the driver is closed)."""
        self.driver.lib.cc_set_exchange(self.driver.ctx, None, None)
