"""gravity_direct on the GPU (gpugrav_gravity_direct): what gravity() runs instead of the tree when fewer
than DIRECT_SUMMATION_THRESHOLD particles are active (src/gravity/accel.c:103-110).  FP64 bit-exact
with the C oracle's restatement of gravdirect.c/force_evaluate_direct, which the CPU tests pin to the
reference's own gravity_direct; here also against that reference build directly where it is present.
TreePM (tabulated short-range factor), isolated, and periodic without PM (Ewald correction)."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from oracle import oracle as O
from oracle import pm_oracle as PMO

pytestmark = pytest.mark.gpu


def _case(kind):
    if kind == "pm":
        ic = ics.zoom_box(log2_half=10, seed=61, pmgrid=64)
    elif kind == "iso":
        ic = ics.hernquist(1500, seed=62)
    else:
        ic = ics.grid_box(n1=10, seed=63, pmgrid=32)
        ic.update(asmth=0.0, rcut=0.0)
    return ic


def _params(ic, **kw):
    return L.make_params(ic["periodic"], box_size=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], softening=tuple(ic["softening"]),
                         **kw)


@pytest.mark.parametrize("kind", ["pm", "iso", "ewald"])
def test_gravity_direct_bitexact(kind, cuda_lib):
    ic = _case(kind)
    op = O.make_params(ic["periodic"], box=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], softening=tuple(ic["softening"]))
    pos = O.wrap(ic["pos"], op)
    a_o, p_o = O.gravity_direct(pos, ic["mass"], ic["softtype"], op)
    with GravityTree(_params(ic)) as t:
        a, p = t.gravity_direct(pos, ic["mass"], ic["softtype"])
    assert np.array_equal(a, a_o) and np.array_equal(p, p_o)
    if kind != "ewald" and O.ref_available():
        r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], ic["periodic"], asmth=ic["asmth"], rcut=ic["rcut"],
                      softening=tuple(ic["softening"]), dump=0, gt=0, direct=1, passes=1)
        o = r["order_end"]
        with GravityTree(_params(ic)) as t:
            a, p = t.gravity_direct(pos[o], ic["mass"][o], ic["softtype"][o])
        assert np.array_equal(a, r["gacc0"]) and np.array_equal(p, r["pot0"])


def test_compute_switches_to_direct_below_threshold(cuda_lib):
    ic = _case("pm")
    n = len(ic["mass"])
    assert n < L.DIRECT_SUMMATION_THRESHOLD
    prm = _params(ic, precision=L.PREC_FP32)
    prm.flags |= L.FLAG_ALLOW_DIRECT_SUMMATION
    op = O.make_params(True, box=1.0, asmth=ic["asmth"], rcut=ic["rcut"], softening=tuple(ic["softening"]))
    pos = O.wrap(ic["pos"], op)
    a_o, p_o = O.gravity_direct(pos, ic["mass"], ic["softtype"], op)
    with GravityTree(prm) as t:
        acc = np.empty((n, 3))
        pot = np.empty(n)
        ni = np.empty(n, np.int32)
        s = t.lib.gpugrav_compute(t._ctx, n, L.ptr(pos), L.ptr(ic["mass"]), L.ptr(ic["softtype"]), None, None, None, 0,
                                  L.ptr(acc), L.ptr(pot), L.ptr(ni), L.MEM_HOST)
        assert s == L.OK
    assert np.array_equal(acc, a_o) and np.array_equal(pot, p_o) and np.all(ni == n)


def test_gravity_direct_edges(cuda_lib):
    ic = _case("iso")
    with GravityTree(_params(ic)) as t:
        a, p = t.gravity_direct(ic["pos"][:1], ic["mass"][:1], ic["softtype"][:1])
        assert np.all(a == 0) and np.all(p == 0)  # one particle: no force (gravdirect.c:65-81)
        st = ic["softtype"].copy()
        st[7] = 9
        with pytest.raises(L.GpuGravError) as e:
            t.gravity_direct(ic["pos"], ic["mass"], st)
        assert e.value.status == L.ERR_INVALID
        # the context walks again after a load and build
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        t.construct_forcetree()
        acc, _, _ = t.gravity_tree()
        assert np.all(np.isfinite(acc))


def test_forcetest_split(cuda_lib):
    """gpugrav_direct_split (FORCETEST, gravtree_forcetest.c:537-620): the total is the Ewald-corrected
    direct sum (bitwise the direct sum of the same box without the TreePM split), the short-range part
    the erfc-cut sum (bitwise gpugrav_direct FULL) with the reference's potential constant, and their
    difference is the long-range force: the reciprocal-space Ewald sum to 1e-5 of its rms, and the
    PM's force to the PM's own accuracy (1.7 % in the CPU restatement of the PM for this clustered
    box; a near-uniform box has so little long-range force that the PM's mesh error dominates it)."""
    ic = ics.zoom_box(log2_half=12, seed=81, pmgrid=64)
    n = len(ic["mass"])
    tg = np.arange(0, n, 3)
    with GravityTree(_params(ic)) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        at, pt, a_s, p_s = t.direct_split(tg)
        a_full, p_full = t.direct(tg)
        pos = O.wrap(ic["pos"], O.make_params(True, asmth=ic["asmth"], rcut=ic["rcut"], softening=tuple(ic["softening"])))
        a_pm, _ = t.pm_periodic(64, pos, ic["mass"])
    assert np.array_equal(a_s, a_full)
    assert np.allclose(p_s - p_full, np.sum(ic["mass"]) * np.pi / ic["asmth"] ** 2, rtol=1e-12, atol=0)
    ew = dict(ic, asmth=0.0, rcut=0.0)
    with GravityTree(_params(ew)) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        a_e, p_e = t.direct(tg)
    assert np.array_equal(at, a_e) and np.array_equal(pt, p_e)
    lr = at - a_s
    scale = np.sqrt(np.mean(np.sum(lr * lr, axis=1)))
    a_k, _ = PMO.longrange_ewald(pos, ic["mass"], ic["box"], ic["asmth"], targets=tg)
    assert np.sqrt(np.mean(np.sum((a_k - lr) ** 2, axis=1))) < 1e-5 * scale
    assert np.sqrt(np.mean(np.sum((a_pm[tg] - lr) ** 2, axis=1))) < 0.03 * scale
