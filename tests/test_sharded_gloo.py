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


def _direct_slice(pos, mass, st, oldacc, slice_, nslices):
    """Softened direct sum for targets [n*s/ns, n*(s+1)/ns) of the full set, zeros elsewhere."""
    p = pos.numpy()
    m = mass.numpy()
    n = len(m)
    a = np.zeros((n, 3))
    pot = np.zeros(n)
    lo, hi = n * slice_ // nslices, n * (slice_ + 1) // nslices
    for i in range(lo, hi):
        d = p - p[i]
        r2 = np.sum(d * d, axis=1) + EPS * EPS
        w = m / (r2 * np.sqrt(r2))
        w[i] = 0.0
        a[i] = np.sum(d * w[:, None], axis=0)
        pot[i] = -np.sum(np.where(np.arange(n) == i, 0.0, m / np.sqrt(r2)))
    return torch.from_numpy(a), torch.from_numpy(pot)


def _particles(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.uniform(0.5, 1.5, n) / n, np.zeros(n, np.uint8)


def _worker(rank, world, port, counts, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from arepo_b200.sharded import ShardedGravity

        pos, mass, st = _particles(sum(counts))
        lo = sum(counts[:rank])
        sl = slice(lo, lo + counts[rank])
        sg = ShardedGravity(walk_slice=_direct_slice)
        acc, pot = sg.compute(torch.from_numpy(pos[sl].copy()), torch.from_numpy(mass[sl].copy()),
                              torch.from_numpy(st[sl].copy()), torch.from_numpy(np.ones(counts[rank], np.float32)))
        np.savez(f"{out_path}.{rank}.npz", acc=acc.numpy(), pot=pot.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("counts", [[37, 50], [20, 33, 25]])
def test_sharded_forces_equal_single_process(counts, tmp_path):
    world = len(counts)
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, _free_port(), counts, out), nprocs=world, join=True, start_method="spawn")
    pos, mass, st = _particles(sum(counts))
    full_acc, full_pot = _direct_slice(torch.from_numpy(pos), torch.from_numpy(mass), None, None, 0, 1)
    lo = 0
    for r, c in enumerate(counts):
        res = np.load(f"{out}.{r}.npz")
        assert res["acc"].shape == (c, 3)
        assert np.array_equal(res["acc"], full_acc.numpy()[lo:lo + c])
        assert np.array_equal(res["pot"], full_pot.numpy()[lo:lo + c])
        lo += c
