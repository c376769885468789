"""One system over G ranks, one process per GPU (torch.distributed, NCCL on GPUs).

Every rank owns a contiguous chunk of the particles (its local arrays). A force computation:

1. one all-gather of the particles packed into 41-byte rows (position, mass, OldAcc, cost, softening
   type): every GPU needs every source,
2. the same tree on every rank (deterministic build from the same particles),
3. each rank walks its own slice of the targets in Peano-Hilbert order: slices of equal cost when
   the caller passes costs (the previous step's interaction counts, what force_assign_cost_values
   feeds the reference's domain decomposition, src/gravity/forcetree.c:945-1010;
   `gpugrav_set_target_slice_cost`), else of equal counts; outputs of other targets are zero,
4. reduce-scatter (sum) of forces, potentials and interaction counts: each rank receives its own
   particles' values (the counts are the next step's costs).

Each target's force is computed by exactly one rank, exactly as in the unsliced walk, so the
result is bitwise identical to the one-GPU computation.  This replaces the reference's
domain-decomposed walk with export/import of targets (src/gravity/gravtree.c:357-707 with
src/utils/generic_comm_helpers2.h) by full replication of the sources, which NVSwitch makes cheap
(2^24 particles are 0.55 GB).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


class ShardedGravity:
    """`compute(pos, mass, softtype, oldacc=None, cost=None)` on this rank's particles (device tensors of
    the process group's device, or CPU tensors with gloo) -> this rank's accelerations, potentials and
    interaction counts.

    `walk_slice(pos, mass, st, oldacc, slice_, nslices, cost) -> (acc, pot, ninter)` computes the forces
    of one target slice for the full particle set (zeros elsewhere); cost (per particle, or None) asks
    for slices of equal cost.  The default uses the GPU library (`GravityTree` on device buffers);
    tests on CPU pass their own."""

    def __init__(self, params=None, device: int | None = None, group=None, walk_slice=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._tree = None
        if walk_slice is None:
            from .gravity import GravityTree

            self._tree = GravityTree(params, device=torch.cuda.current_device() if device is None else device)
            self._stream = torch.cuda.current_stream()
            self._tree.set_stream(self._stream.cuda_stream)
            walk_slice = self._gpu_walk_slice
        self.walk_slice = walk_slice

    def close(self):
        if self._tree is not None:
            self._tree.close()
            self._tree = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- the library on device buffers ----
    def _gpu_walk_slice(self, pos, mass, st, oldacc, slice_, nslices, cost=None):
        from . import _lib as L

        t = self._tree
        n = mass.shape[0]
        acc = torch.empty((n, 3), dtype=torch.float64, device=pos.device)
        pot = torch.empty(n, dtype=torch.float64, device=pos.device)
        ni = torch.empty(n, dtype=torch.int32, device=pos.device)
        if cost is None:
            t.set_target_slice(slice_, nslices)
        else:
            t.set_target_slice_cost(slice_, nslices, cost.contiguous(), mem=L.MEM_DEVICE)
        s = t.lib.gpugrav_compute(t._ctx, n, L.ptr(pos), L.ptr(mass), L.ptr(st),
                                  None if oldacc is None else L.ptr(oldacc), None, None, 0, L.ptr(acc), L.ptr(pot),
                                  L.ptr(ni), L.MEM_DEVICE)
        if s != L.OK:
            raise L.GpuGravError(s, t.lib.gpugrav_last_error(t._ctx).decode())
        return acc, pot, ni

    # ---- one force computation ----
    def _gather(self, x, counts, maxn):
        """All ranks' rows of x (first dimension), in rank order."""
        pad = torch.zeros((maxn,) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        pad[: x.shape[0]] = x
        out = torch.empty((self.world * maxn,) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        dist.all_gather_into_tensor(out, pad, group=self.group)
        return torch.cat([out[r * maxn: r * maxn + counts[r]] for r in range(self.world)])

    def _scatter_sum(self, full, counts, maxn):
        """Sum over ranks of `full` (all particles, rank order); each rank gets its own rows."""
        chunks = torch.zeros((self.world * maxn,) + tuple(full.shape[1:]), dtype=full.dtype, device=full.device)
        off = 0
        for r in range(self.world):
            chunks[r * maxn: r * maxn + counts[r]] = full[off: off + counts[r]]
            off += counts[r]
        out = torch.empty((maxn,) + tuple(full.shape[1:]), dtype=full.dtype, device=full.device)
        dist.reduce_scatter_tensor(out, chunks, op=dist.ReduceOp.SUM, group=self.group)
        return out[: counts[self.rank]]

    ROW = 41  # bytes per particle in the all-gather: 3 x f64 position, f64 mass, f32 OldAcc, f32 cost, u8 type

    @staticmethod
    def _pack(pos, mass, st, oldacc, cost):
        n = mass.shape[0]
        z = torch.zeros(n, dtype=torch.float32, device=pos.device)
        cols = [pos.contiguous().view(torch.uint8).reshape(n, 24), mass.contiguous().view(torch.uint8).reshape(n, 8),
                (z if oldacc is None else oldacc.to(torch.float32).contiguous()).view(torch.uint8).reshape(n, 4),
                (z if cost is None else cost.to(torch.float32).contiguous()).view(torch.uint8).reshape(n, 4),
                st.contiguous().view(torch.uint8).reshape(n, 1)]
        return torch.cat(cols, dim=1)

    @staticmethod
    def _unpack(rows):
        n = rows.shape[0]
        pos = rows[:, 0:24].contiguous().view(torch.float64).reshape(n, 3)
        mass = rows[:, 24:32].contiguous().view(torch.float64).reshape(n)
        old = rows[:, 32:36].contiguous().view(torch.float32).reshape(n)
        cost = rows[:, 36:40].contiguous().view(torch.float32).reshape(n)
        st = rows[:, 40].contiguous()
        return pos, mass, st, old, cost

    def compute(self, pos, mass, softtype, oldacc=None, cost=None):
        """-> (acc, pot, ninter) of this rank's particles.  cost (this rank's particles, e.g. the ninter of
        the previous step) balances the slices by cost; every rank passes costs or none does."""
        n_local = torch.tensor([mass.shape[0]], dtype=torch.int64, device=pos.device)
        all_n = torch.empty(self.world, dtype=torch.int64, device=pos.device)
        dist.all_gather_into_tensor(all_n, n_local, group=self.group)
        counts = [int(v) for v in all_n.tolist()]
        maxn = max(counts)
        rows = self._gather(self._pack(pos, mass, softtype, oldacc, cost), counts, maxn)
        fpos, fmass, fst, fold, fcost = self._unpack(rows)
        acc, pot, ni = self.walk_slice(fpos, fmass, fst, None if oldacc is None else fold, self.rank, self.world,
                                       None if cost is None else fcost)
        return (self._scatter_sum(acc, counts, maxn), self._scatter_sum(pot, counts, maxn),
                self._scatter_sum(ni.to(torch.int64), counts, maxn))
