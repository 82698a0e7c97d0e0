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
"""
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
