"""Host logic of the sharded multi-GPU force computation (arepo_b200/sharded.py) on CPU ranks
with the gloo backend: particles owned in unequal chunks by 2 or 3 ranks are all-gathered, every
rank computes one target slice of the full set, and the reduce-scatter returns each rank exactly
the forces of its own particles -- bitwise equal to one process computing all targets.

The per-slice force here is a softened FP64 direct sum in numpy (the library's GPU walk is
covered by tests/test_gpu_slices.py, which checks that the slices of the real walk sum to the
unsliced walk bit for bit)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

EPS = 0.05


def _bounds(n, slice_, nslices, cost):
    """Target range of a slice: equal counts, or equal cost (the library's rule: slice s starts at the
    first target whose exclusive cost prefix reaches s/nslices of the total)."""
    if cost is None:
        return n * slice_ // nslices, n * (slice_ + 1) // nslices
    c = cost.numpy().astype(np.float64)
    ex = np.concatenate([[0.0], np.cumsum(c)[:-1]])
    tot = c.sum()
    b = [0 if s == 0 else n if s == nslices else int(np.searchsorted(ex, tot * s / nslices, side="left"))
         for s in (slice_, slice_ + 1)]
    return b[0], b[1]


def _direct_slice(pos, mass, st, oldacc, slice_, nslices, cost=None):
    """Softened direct sum for the targets of one slice of the full set, zeros elsewhere; the cost of
    a target is its index + 1 (a stand-in for interaction counts)."""
    p = pos.numpy()
    m = mass.numpy()
    n = len(m)
    a = np.zeros((n, 3))
    pot = np.zeros(n)
    ni = np.zeros(n, np.int32)
    lo, hi = _bounds(n, slice_, nslices, cost)
    for i in range(lo, hi):
        d = p - p[i]
        r2 = np.sum(d * d, axis=1) + EPS * EPS
        w = m / (r2 * np.sqrt(r2))
        w[i] = 0.0
        a[i] = np.sum(d * w[:, None], axis=0)
        pot[i] = -np.sum(np.where(np.arange(n) == i, 0.0, m / np.sqrt(r2)))
        ni[i] = i + 1
    return torch.from_numpy(a), torch.from_numpy(pot), torch.from_numpy(ni)


def _particles(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.uniform(0.5, 1.5, n) / n, np.zeros(n, np.uint8)


def _worker(rank, world, port, counts, out_path, with_cost=False):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from arepo_b200.sharded import ShardedGravity

        pos, mass, st = _particles(sum(counts))
        lo = sum(counts[:rank])
        sl = slice(lo, lo + counts[rank])
        sg = ShardedGravity(walk_slice=_direct_slice)
        args = (torch.from_numpy(pos[sl].copy()), torch.from_numpy(mass[sl].copy()), torch.from_numpy(st[sl].copy()),
                torch.from_numpy(np.ones(counts[rank], np.float32)))
        acc, pot, ni = sg.compute(*args)
        if with_cost:  # the next step balances the slices by this step's counts
            acc, pot, ni = sg.compute(*args, cost=ni)
        np.savez(f"{out_path}.{rank}.npz", acc=acc.numpy(), pot=pot.numpy(), ni=ni.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("with_cost", [False, True])
@pytest.mark.parametrize("counts", [[37, 50], [20, 33, 25]])
def test_sharded_forces_equal_single_process(counts, with_cost, tmp_path):
    world = len(counts)
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, _free_port(), counts, out, with_cost), nprocs=world, join=True,
                       start_method="spawn")
    pos, mass, st = _particles(sum(counts))
    full_acc, full_pot, full_ni = _direct_slice(torch.from_numpy(pos), torch.from_numpy(mass), None, None, 0, 1)
    lo = 0
    for r, c in enumerate(counts):
        res = np.load(f"{out}.{r}.npz")
        assert res["acc"].shape == (c, 3)
        assert np.array_equal(res["acc"], full_acc.numpy()[lo:lo + c])
        assert np.array_equal(res["pot"], full_pot.numpy()[lo:lo + c])
        assert np.array_equal(res["ni"], full_ni.numpy()[lo:lo + c])
        lo += c
