"""The sharded driver (arepo_b200/sharded.py) on the GPU with NCCL, one rank in this process: the
particles go through the packed all-gather, the library walks the rank's slice on torch's default
stream, and the forces come back through the reduce-scatter.  No host synchronisation between the
calls, so the library's work must be ordered after torch's packing and gather on the same stream.
Bitwise the same as the library called directly on the same particles (FP32 group walk: the
Barnes-Hut pass, then relative passes with OldAcc, equal-count and cost-balanced slices)."""
import datetime

import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_one_rank(cuda_lib):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    store = dist.HashStore()
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    yield dist
    dist.destroy_process_group()


def test_sharded_one_rank_matches_library(nccl_one_rank):
    import torch

    from arepo_b200.sharded import ShardedGravity

    ic = ics.zoom_box(log2_half=18, seed=91, pmgrid=128)
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(ic["pos"].copy()).to(dev)
    mass_d = torch.from_numpy(ic["mass"].copy()).to(dev)
    st_d = torch.from_numpy(ic["softtype"].copy()).to(dev)
    prm = ics.params_for(ic, precision=L.PREC_FP32)
    with ShardedGravity(prm, device=0) as sg:
        acc_bh, _, _ = sg.compute(pos_d, mass_d, st_d, None)
        acc_bh = acc_bh.cpu().numpy()
        old = np.linalg.norm(acc_bh, axis=1).astype(np.float32)  # OldAcc of both paths
        old_d = torch.from_numpy(old).to(dev)
        prm.err_tol_theta = 0.0
        prm.err_tol_force_acc = 6e-5
        sg._tree.set_params(prm)
        acc1, pot1, ni1 = sg.compute(pos_d, mass_d, st_d, old_d)
        acc2, pot2, ni2 = sg.compute(pos_d, mass_d, st_d, old_d, ni1.to(torch.float32))
        torch.cuda.synchronize()
        acc1, pot1, ni1, acc2 = (x.cpu().numpy() for x in (acc1, pot1, ni1, acc2))
    # the same particles through the library directly (host buffers)
    prm_bh = ics.params_for(ic, precision=L.PREC_FP32)
    with GravityTree(prm_bh) as t:
        n = len(ic["mass"])
        a = np.empty((n, 3))
        p = np.empty(n)
        ni = np.empty(n, np.int32)
        s = t.lib.gpugrav_compute(t._ctx, n, L.ptr(ic["pos"]), L.ptr(ic["mass"]), L.ptr(ic["softtype"]), None, None,
                                  None, 0, L.ptr(a), L.ptr(p), L.ptr(ni), L.MEM_HOST)
        assert s == L.OK
        assert np.array_equal(a, acc_bh)
        t.set_params(prm)
        s = t.lib.gpugrav_compute(t._ctx, n, L.ptr(ic["pos"]), L.ptr(ic["mass"]), L.ptr(ic["softtype"]), L.ptr(old),
                                  None, None, 0, L.ptr(a), L.ptr(p), L.ptr(ni), L.MEM_HOST)
        assert s == L.OK
    assert np.array_equal(a, acc1) and np.array_equal(p, pot1) and np.array_equal(ni, ni1)
    assert np.array_equal(a, acc2)  # one slice: cost balancing changes nothing


def test_set_stream_default_is_ordered(cuda_lib):
    """A torch default-stream handle (0) is taken as the legacy default stream, not as 'own stream'."""
    import torch

    ic = ics.grid_box(n1=16, seed=92, pmgrid=32)
    with GravityTree(ics.params_for(ic, precision=L.PREC_FP32)) as t:
        t.set_stream(torch.cuda.current_stream().cuda_stream)
        dev = torch.device("cuda", 0)
        n = len(ic["mass"])
        for _ in range(3):
            # inputs written by torch right before the call, outputs read right after, no host sync
            pos_d = torch.from_numpy(ic["pos"].copy()).to(dev) * 1.0
            mass_d = torch.from_numpy(ic["mass"].copy()).to(dev) * 1.0
            st_d = torch.from_numpy(ic["softtype"].copy()).to(dev)
            acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
            pot = torch.empty(n, dtype=torch.float64, device=dev)
            ni = torch.empty(n, dtype=torch.int32, device=dev)
            s = t.lib.gpugrav_compute(t._ctx, n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), None, None, None, 0,
                                      L.ptr(acc), L.ptr(pot), L.ptr(ni), L.MEM_DEVICE)
            assert s == L.OK
            total = torch.isfinite(acc).all() & (ni > 0).all()
            assert bool(total.cpu())
