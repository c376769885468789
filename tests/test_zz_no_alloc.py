"""gpugrav_direct_noalloc: the direct summation for callers that cannot allocate
device memory (their GPU memory belongs to their own pool allocator, or they
cannot take the device-wide synchronisation of cudaMalloc mid-step).

Checked through the C ABI against the context-based gpugrav_direct on two calls
in a row (different targets and modes, so that the second call runs over the
first call's leftovers in the shared scratch array), within the tolerance of the
other direct-sum test.  Kept in a file collected last."""
import ctypes as C

import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200.gravity import GravityTree
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _params(p):
    return L.make_params(periodic=p["periodic"], box_size=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                         rcut_cells=p["rcut_cells"], softening=tuple(p["softening"]), err_tol_theta=p["theta"],
                         err_tol_force_acc=p["erracc"], top_node_factor=p["tnf"], multiple_domains=p["mdom"])


@pytest.mark.parametrize("name", ["grid16_pm", "hernquist2048_iso"])
def test_direct_noalloc_matches_direct(name, cuda_lib):
    import torch

    g = load_golden(name)
    prm = _params(g["params"])
    n = len(g["mass"])
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(g["pos"])).to(dev)
    mass_d = torch.from_numpy(np.ascontiguousarray(g["mass"])).to(dev)
    st_d = torch.from_numpy(np.ascontiguousarray(g["softtype"])).to(dev)
    calls = [(np.arange(0, n, 5), L.DIRECT_FULL), (np.arange(3, n, 7)[:300], L.DIRECT_CUT)]
    with GravityTree(prm) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        for tg, mode in calls:
            ref_acc, ref_pot = t.direct(tg, cut=(mode == L.DIRECT_CUT))
            tg_d = torch.from_numpy(tg).to(dev)
            tpos = pos_d[tg_d].contiguous()
            tst = st_d[tg_d].contiguous()
            acc = torch.full((len(tg), 3), float("nan"), dtype=torch.float64, device=dev)
            pot = torch.full((len(tg),), float("nan"), dtype=torch.float64, device=dev)
            s = cuda_lib.gpugrav_direct_noalloc(0, C.byref(prm), n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), len(tg),
                                                L.ptr(tpos), L.ptr(tst), mode, L.ptr(acc), L.ptr(pot), None)
            assert s == L.OK
            torch.cuda.synchronize()
            a, p = acc.cpu().numpy(), pot.cpu().numpy()
            # the same FP64 pair sum as gpugrav_direct, summed in another order
            assert np.max(np.abs(a - ref_acc)) < 1e-11 * np.max(np.abs(ref_acc))
            assert np.max(np.abs(p - ref_pot)) < 1e-11 * np.max(np.abs(ref_pot))


def test_direct_noalloc_rejects_oversized_requests(cuda_lib):
    import torch

    g = load_golden("grid16_pm")
    prm = _params(g["params"])
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(g["pos"])).to(dev)
    mass_d = torch.from_numpy(np.ascontiguousarray(g["mass"])).to(dev)
    st_d = torch.from_numpy(np.ascontiguousarray(g["softtype"])).to(dev)
    acc = torch.empty((4097, 3), dtype=torch.float64, device=dev)
    s = cuda_lib.gpugrav_direct_noalloc(0, C.byref(prm), len(g["mass"]), L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), 4097,
                                        L.ptr(pos_d), L.ptr(st_d), L.DIRECT_FULL, L.ptr(acc), None, None)
    assert s == L.ERR_TOO_LARGE
    assert b"4096" in cuda_lib.gpugrav_status_string(s)
