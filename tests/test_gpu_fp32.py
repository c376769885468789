"""The FP32 group walk: accuracy against FP64 direct summation, compared with the
FP64 parity walk (the reference's own decisions) on the same particles.

The group walk accepts a node only if every target of the group would accept it,
so its tree-approximation error must not exceed the parity walk's; FP32
arithmetic with FP64 separations adds a rounding error far below 1e-4."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _run(ic, precision, targets):
    prm = ics.params_for(ic, precision=precision)
    with GravityTree(prm) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        d_cut, _ = t.direct(targets, cut=True)
    return acc, pot, ni, d_cut


def _err(acc, ref):
    dn = np.linalg.norm(ref, axis=1)
    e = np.linalg.norm(acc - ref, axis=1)
    scale = np.sqrt(np.mean(dn * dn))
    return float(np.sqrt(np.mean((e / np.maximum(dn, 1e-300)) ** 2))), float(np.sqrt(np.mean((e / scale) ** 2)))


CASES = {
    "grid32": lambda: ics.grid_box(n1=32, seed=1001, pmgrid=64),
    "hernquist": lambda: ics.hernquist(1 << 16, seed=1002),
    "zoom": lambda: ics.zoom_box(log2_half=15, seed=1004, pmgrid=128),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_walk_at_least_as_accurate_as_parity_walk(name, cuda_lib):
    ic = CASES[name]()
    n = len(ic["mass"])
    tg = np.sort(np.random.default_rng(5).choice(n, 2048, replace=False))
    a64, _, n64, d = _run(ic, L.PREC_FP64, tg)
    a32, _, n32, _ = _run(ic, L.PREC_FP32, tg)
    rel64, glob64 = _err(a64[tg], d)
    rel32, glob32 = _err(a32[tg], d)
    # conservative group decisions: no less accurate than per-target decisions (FP32 rounding slack)
    assert glob32 <= glob64 * 1.02 + 2e-5, (glob32, glob64)
    assert rel32 <= rel64 * 1.02 + 2e-5, (rel32, rel64)
    assert n32.sum() >= n64.sum()
    assert np.all(np.isfinite(a32))


def test_fp32_walk_matches_fp64_walk_with_tight_criterion(cuda_lib):
    """With a very tight relative criterion both walks converge to the direct sum; FP32
    rounding with FP64 separations stays below 1e-5 relative."""
    ic = ics.grid_box(n1=24, seed=3, pmgrid=48)
    prm64 = ics.params_for(ic, precision=L.PREC_FP64, err_tol_force_acc=1e-7)
    prm32 = ics.params_for(ic, precision=L.PREC_FP32, err_tol_force_acc=1e-7)
    with GravityTree(prm64) as t:
        a64, _, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
    with GravityTree(prm32) as t:
        a32, p32, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
    scale = np.sqrt(np.mean(np.sum(a64 * a64, axis=1)))
    err = np.linalg.norm(a32 - a64, axis=1) / scale
    assert np.sqrt(np.mean(err ** 2)) < 1e-5
    assert np.all(np.isfinite(p32))


@pytest.mark.parametrize("name", ["grid16_pm", "hernquist2048_iso", "mix1500_pm"])
def test_fp32_walk_on_golden_inputs(name, cuda_lib):
    g = load_golden(name)
    p = g["params"]
    ic = dict(pos=g["pos"], mass=g["mass"], softtype=g["softtype"], periodic=p["periodic"], box=p["box"],
              asmth=p["asmth"], rcut=p["rcut"], softening=tuple(p["softening"]))
    tg = np.arange(len(g["mass"]))
    a64, _, _, d = _run(ic, L.PREC_FP64, tg)
    a32, _, _, _ = _run(ic, L.PREC_FP32, tg)
    _, glob64 = _err(a64, d)
    _, glob32 = _err(a32, d)
    assert glob32 <= glob64 * 1.02 + 2e-5
    # and the FP64 path is the reference's own result
    assert np.array_equal(a64[g["order"]], g["acc1"])


def test_fp32_walk_without_potential_gives_same_forces(cuda_lib):
    ic = ics.zoom_box(log2_half=13, seed=11, pmgrid=64)
    prm = ics.params_for(ic, precision=L.PREC_FP32)
    with GravityTree(prm) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        t.construct_forcetree()
        a1, p1, n1 = t.gravity_tree()
        a2, p2, n2 = t.gravity_tree(want_pot=False)
    assert p2 is None and np.all(np.isfinite(p1))
    assert np.array_equal(a1, a2) and np.array_equal(n1, n2)


def test_fp32_walk_isolated_outliers_stay_local(cuda_lib):
    """Untruncated Plummer sphere: key-order neighbours in the sparse outskirts can lie on both
    sides of the core. Their group box then contains the core, and the box test alone would open
    it down to single particles for every target of the group (interaction counts of order N).
    The per-target vote keeps every target's list close to its own walk's."""
    ic = ics.plummer(1 << 17, seed=9)
    n = len(ic["mass"])
    tg = np.sort(np.random.default_rng(6).choice(n, 2048, replace=False))
    a64, _, n64, d = _run(ic, L.PREC_FP64, tg)
    a32, _, n32, _ = _run(ic, L.PREC_FP32, tg)
    assert n32.max() < 0.3 * n, n32.max()
    assert n32.sum() >= n64.sum()
    rel64, glob64 = _err(a64[tg], d)
    rel32, glob32 = _err(a32[tg], d)
    assert glob32 <= glob64 * 1.02 + 2e-5, (glob32, glob64)


def test_fp32_walk_multiple_node_softening(cuda_lib):
    """MULTIPLE_NODE_SOFTENING with two very different softenings: nodes with large-softening mass
    near small-softening targets are listed per type in the FP32 walk; its error against the direct
    sum is no larger than the FP64 parity walk's (which follows the reference per target)."""
    rng = np.random.default_rng(41)
    n = 40000
    st = (np.arange(n) >= n // 3).astype(np.uint8)
    pos = np.where(st[:, None] == 0, np.mod(0.5 + 0.08 * rng.normal(size=(n, 3)), 1.0),
                   np.mod(0.5 + 0.03 * rng.normal(size=(n, 3)), 1.0))
    mass = np.where(st == 0, 8.0, 1.0) / n
    a = 1.25 / 128
    ic = dict(pos=pos, mass=mass, softtype=st, softening=(0.004, 0.0004), periodic=True, box=1.0, asmth=a,
              rcut=4.5 * a)
    tg = np.sort(rng.choice(n, 2048, replace=False))
    out = {}
    for prec in (L.PREC_FP64, L.PREC_FP32):
        prm = ics.params_for(ic, precision=prec)
        prm.flags = L.FLAG_MULTIPLE_NODE_SOFTENING
        with GravityTree(prm) as t:
            acc, _, ni, _ = t.compute_grav_accelerations(pos, mass, st)
            d, _ = t.direct(tg, cut=True)
        out[prec] = (acc, ni, d)
    d = out[L.PREC_FP64][2]
    rel64, glob64 = _err(out[L.PREC_FP64][0][tg], d)
    rel32, glob32 = _err(out[L.PREC_FP32][0][tg], d)
    assert glob32 <= glob64 * 1.02 + 2e-5, (glob32, glob64)
    assert rel32 <= rel64 * 1.02 + 2e-5, (rel32, rel64)


@pytest.mark.parametrize("name", ["zoom", "hernquist"])
def test_fp64_group_walk_is_the_fp32_walk_in_double(name, cuda_lib):
    """GPUGRAV_PREC_FP64_GROUP runs the FP32 walk's algorithm (same groups, same opening decisions, same
    interaction lists) with FP64 arithmetic: it differs from the FP32 walk by FP32 rounding only, and
    is no less accurate than the FP64 parity walk against the direct sum."""
    ic = CASES[name]()
    n = len(ic["mass"])
    tg = np.sort(np.random.default_rng(6).choice(n, 2048, replace=False))
    a32, _, n32, d = _run(ic, L.PREC_FP32, tg)
    ag, _, ng, _ = _run(ic, L.PREC_FP64_GROUP, tg)
    a64, _, _, _ = _run(ic, L.PREC_FP64, tg)
    scale = np.sqrt(np.mean(np.sum(ag * ag, axis=1)))
    assert np.sqrt(np.mean(np.sum((a32 - ag) ** 2, axis=1))) / scale < 1e-5
    assert abs(int(ng.sum()) - int(n32.sum())) <= 1e-5 * int(n32.sum())  # pairs at Rcut may round either way
    _, glob64 = _err(a64[tg], d)
    _, globg = _err(ag[tg], d)
    assert globg <= glob64 * 1.02 + 2e-5, (globg, glob64)
