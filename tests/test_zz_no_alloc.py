"""gpugrav_direct_noalloc: the direct summation for callers that cannot allocate
device memory when they call it -- a code whose GPU memory belongs to its own
pool allocator (reserved once at start-up), or one that cannot take the
device-wide synchronisation of cudaMalloc/cudaFree in the middle of a step.

Checked through the C ABI against the context-based gpugrav_direct and against
the C oracle's direct sum, on two calls in a row (different targets and modes, so
that the second call runs over the first call's leftovers in the shared scratch
array), within the tolerance of the other direct-sum tests (1e-11 of the largest
value: CUDA's and glibc's erfc differ by a few ulp and the summation order
differs).  Kept in a file collected last."""
import ctypes as C

import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200.gravity import GravityTree
from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _params(p):
    return L.make_params(periodic=p["periodic"], box_size=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                         rcut_cells=p["rcut_cells"], softening=tuple(p["softening"]), err_tol_theta=p["theta"],
                         err_tol_force_acc=p["erracc"], top_node_factor=p["tnf"], multiple_domains=p["mdom"])


def _oparams(p):
    return O.make_params(p["periodic"], box=p["box"], asmth=p["asmth"], rcut=p["rcut"], rcut_cells=p["rcut_cells"],
                         theta=p["theta"], erracc=p["erracc"], softening=tuple(p["softening"]), mdom=p["mdom"], tnf=p["tnf"])


def _call(lib, prm, pos_d, mass_d, st_d, tpos, tst, mode, stream=None):
    import torch

    nt = tpos.shape[0]
    acc = torch.full((nt, 3), float("nan"), dtype=torch.float64, device=pos_d.device)
    pot = torch.full((nt,), float("nan"), dtype=torch.float64, device=pos_d.device)
    s = lib.gpugrav_direct_noalloc(0, C.byref(prm), mass_d.shape[0], L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), nt,
                                   L.ptr(tpos), L.ptr(tst), mode, L.ptr(acc), L.ptr(pot), stream)
    return s, acc, pot


def _close(a, b):
    return np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b))


@pytest.mark.parametrize("name", ["grid16_pm", "hernquist2048_iso"])
def test_direct_noalloc_matches_direct_and_oracle(name, cuda_lib):
    import torch

    g = load_golden(name)
    prm = _params(g["params"])
    op = _oparams(g["params"])
    n = len(g["mass"])
    wpos = O.wrap(g["pos"], op)
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(wpos)).to(dev)
    mass_d = torch.from_numpy(np.ascontiguousarray(g["mass"])).to(dev)
    st_d = torch.from_numpy(np.ascontiguousarray(g["softtype"])).to(dev)
    calls = [(np.arange(0, n, 5), L.DIRECT_FULL), (np.arange(3, n, 7)[:300], L.DIRECT_CUT)]
    with GravityTree(prm) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        for tg, mode in calls:
            ref_acc, ref_pot = t.direct(tg, cut=(mode == L.DIRECT_CUT))
            tg_d = torch.from_numpy(tg).to(dev)
            s, acc, pot = _call(cuda_lib, prm, pos_d, mass_d, st_d, pos_d[tg_d].contiguous(), st_d[tg_d].contiguous(), mode)
            assert s == L.OK
            torch.cuda.synchronize()
            a, p = acc.cpu().numpy(), pot.cpu().numpy()
            assert _close(a, ref_acc) and _close(p, ref_pot)
            if mode == L.DIRECT_FULL:
                # the C oracle's direct sum (gravity_forcetest_evaluate's pair sum) on the same particles
                o_acc, o_pot = O.direct(wpos, g["mass"], g["softtype"], op, tg)
                assert _close(a, o_acc) and _close(p, o_pot)


def test_direct_noalloc_few_sources_side_stream(cuda_lib):
    """5 sources (most of the 32 source chunks are empty) on a non-default stream, twice in a row."""
    import torch

    g = load_golden("hernquist2048_iso")
    p = g["params"]
    prm, op = _params(p), _oparams(p)
    rng = np.random.default_rng(5)
    src = rng.choice(len(g["mass"]), 5, replace=False)
    pos, mass, st = g["pos"][src].copy(), g["mass"][src].copy(), g["softtype"][src].copy()
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(pos).to(dev)
    mass_d = torch.from_numpy(mass).to(dev)
    st_d = torch.from_numpy(st).to(dev)
    side = torch.cuda.Stream(device=dev)
    o_acc, o_pot = O.direct(pos, mass, st, op, np.arange(5))
    for _ in range(2):
        with torch.cuda.stream(side):
            s, acc, pot = _call(cuda_lib, prm, pos_d, mass_d, st_d, pos_d, st_d, L.DIRECT_FULL, stream=side.cuda_stream)
        assert s == L.OK
        side.synchronize()
        assert _close(acc.cpu().numpy(), o_acc) and _close(pot.cpu().numpy(), o_pot)


def test_direct_noalloc_bad_softening_type_gives_nan(cuda_lib):
    import torch

    g = load_golden("grid16_pm")
    prm = _params(g["params"])
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(O.wrap(g["pos"], _oparams(g["params"])))).to(dev)
    mass_d = torch.from_numpy(np.ascontiguousarray(g["mass"])).to(dev)
    st_d = torch.from_numpy(np.ascontiguousarray(g["softtype"])).to(dev)
    tpos = pos_d[:8].contiguous()
    tst = st_d[:8].clone()
    tst[2] = 200  # no softening length for this type: that target's outputs are NaN
    s, acc, pot = _call(cuda_lib, prm, pos_d, mass_d, st_d, tpos, tst, L.DIRECT_FULL)
    assert s == L.OK
    torch.cuda.synchronize()
    a, p = acc.cpu().numpy(), pot.cpu().numpy()
    assert np.all(np.isnan(a[2])) and np.isnan(p[2])
    assert np.all(np.isfinite(np.delete(a, 2, axis=0))) and np.all(np.isfinite(np.delete(p, 2)))
    bad = st_d.clone()
    bad[11] = 17  # a source of an unknown type poisons every pair it enters (FULL mode: all of them)
    s, acc, pot = _call(cuda_lib, prm, pos_d, mass_d, bad, tpos, st_d[:8].contiguous(), L.DIRECT_FULL)
    assert s == L.OK
    torch.cuda.synchronize()
    assert np.all(np.isnan(acc.cpu().numpy())) and np.all(np.isnan(pot.cpu().numpy()))


def test_direct_noalloc_rejects_oversized_and_invalid_requests(cuda_lib):
    import torch

    g = load_golden("grid16_pm")
    prm = _params(g["params"])
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(np.ascontiguousarray(g["pos"])).to(dev)
    mass_d = torch.from_numpy(np.ascontiguousarray(g["mass"])).to(dev)
    st_d = torch.from_numpy(np.ascontiguousarray(g["softtype"])).to(dev)
    acc = torch.empty((4097, 3), dtype=torch.float64, device=dev)
    n = len(g["mass"])
    s = cuda_lib.gpugrav_direct_noalloc(0, C.byref(prm), n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), 4097,
                                        L.ptr(pos_d), L.ptr(st_d), L.DIRECT_FULL, L.ptr(acc), None, None)
    assert s == L.ERR_TOO_LARGE
    assert b"4096" in cuda_lib.gpugrav_status_string(s)
    # the periodic pure-tree mode (asmth == 0) needs the Ewald tables: refused
    ew = _params(dict(g["params"], asmth=0.0, rcut=0.0))
    s = cuda_lib.gpugrav_direct_noalloc(0, C.byref(ew), n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), 4,
                                        L.ptr(pos_d), L.ptr(st_d), L.DIRECT_FULL, L.ptr(acc), None, None)
    assert s == L.ERR_INVALID
    # parameters are checked like gpugrav_create's: rcut <= 0 with the TreePM split is refused
    bad = _params(dict(g["params"], rcut=0.0))
    s = cuda_lib.gpugrav_direct_noalloc(0, C.byref(bad), n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(st_d), 4,
                                        L.ptr(pos_d), L.ptr(st_d), L.DIRECT_CUT, L.ptr(acc), None, None)
    assert s == L.ERR_INVALID
