"""Walks of an active subset of the particles (gpugrav_walk_targets): gravity_tree(timebin)'s
TargetList (src/gravity/gravtree.c:494-520) with the tree holding every particle.

FP64: each active target's acceleration, potential and interaction count are bit-identical to the
walk of every particle, hence to the reference's own output (golden fixtures) and to the C oracle's
per-target walk.  FP32: groups of consecutive active targets; accuracy against the FP64 direct sum no
worse than the FP64 parity walk's on the same targets (the bar of the other FP32 tests)."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from conftest import GOLDEN_CASES, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _gpu_params(p, precision=L.PREC_FP64):
    return L.make_params(periodic=p["periodic"], box_size=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                         rcut_cells=p["rcut_cells"], softening=tuple(p["softening"]), err_tol_theta=p["theta"],
                         err_tol_force_acc=p["erracc"], top_node_factor=p["tnf"], multiple_domains=p["mdom"],
                         precision=precision, multiple_node_softening=p.get("mns", False))


def _active(n, frac, seed):
    rng = np.random.default_rng(seed)
    return rng.permutation(n)[: max(1, int(frac * n))].astype(np.int32)  # caller indices, unsorted


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fp64_active_walk_bitexact_with_reference(name, cuda_lib):
    g = load_golden(name)
    order = g["order"]  # order[sorted position] = caller index
    n = len(order)
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    prm = _gpu_params(g["params"])
    act = _active(n, 0.1, 11)
    with GravityTree(prm) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree(topnodes=g["top"])
        acc, pot, ni = t.gravity_tree_targets(act)
        assert np.array_equal(acc, g["acc0"][inv[act]])
        assert np.array_equal(pot, g["pot0"][inv[act]])
        assert np.array_equal(ni, g["ninter0"][inv[act]])
        oldacc = np.empty(n, np.float32)
        oldacc[order] = g["oldacc0"]
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        acc, pot, ni = t.gravity_tree_targets(act, oldacc)
        assert np.array_equal(acc, g["acc1"][inv[act]])
        assert np.array_equal(pot, g["pot1"][inv[act]])
        assert np.array_equal(ni, g["ninter1"][inv[act]])


def test_fp64_active_walk_matches_oracle_per_target_walk(cuda_lib):
    ic = ics.zoom_box(log2_half=14, seed=21, pmgrid=64)
    soft = tuple(ic["softening"])
    op = O.make_params(True, box=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], softening=soft)
    ref = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], op, passes=1)
    perm = ref["perm"]  # sorted position -> caller index
    n = len(perm)
    act_sorted = np.sort(np.random.default_rng(12).choice(n, n // 10, replace=False))
    oldacc_sorted = ref["oldacc0"]
    op.theta = 0.0
    o_acc, o_pot, o_ni = O.walk(ref["tree"], ref["pos_sorted"], ref["mass_sorted"], ref["st_sorted"], oldacc_sorted, op,
                                targets=act_sorted)
    prm = ics.params_for(ic, precision=L.PREC_FP64)
    oldacc = np.empty(n, np.float32)
    oldacc[perm] = oldacc_sorted
    with GravityTree(prm) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        t.construct_forcetree()
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        acc, pot, ni = t.gravity_tree_targets(perm[act_sorted][::-1].copy(), oldacc)  # any order
    assert np.array_equal(acc[::-1], o_acc)
    assert np.array_equal(pot[::-1], o_pot)
    assert np.array_equal(ni[::-1], o_ni)


@pytest.mark.parametrize("case", ["zoom", "hernquist", "zoom_background"])
def test_fp32_active_walk_accuracy(case, cuda_lib):
    """FP32 walk of an active subset, never less accurate than the FP64 per-target walk of the same
    subset.  zoom_background: the uniform particles only, which follow each other in key order on both
    sides of the dense core (the group table cuts them between cells)."""
    ic = ics.zoom_box(log2_half=15, seed=1004, pmgrid=128) if case != "hernquist" else ics.hernquist(1 << 16, seed=1002)
    n = len(ic["mass"])
    act = _active(n, 0.1, 13) if case != "zoom_background" else np.arange(n // 2, dtype=np.int32)
    res = {}
    for prec in (L.PREC_FP64, L.PREC_FP32):
        prm = ics.params_for(ic, precision=prec)
        with GravityTree(prm) as t:
            a_full, _, _, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
            prm.err_tol_theta = 0.0  # relative criterion, as the second pass of a_full
            t.set_params(prm)
            acc, pot, ni = t.gravity_tree_targets(act, oldacc)
            if prec == L.PREC_FP64:
                d, _ = t.direct(act.astype(np.int64), cut=True)
                assert np.array_equal(acc, a_full[act])  # same walk per target
            else:
                # after an active walk, a walk of every particle is the plain walk again
                a_again, _, _ = t.gravity_tree(oldacc)
                assert np.array_equal(a_again, a_full)
        res[prec] = (acc, ni)
    dn = np.linalg.norm(d, axis=1)
    scale = np.sqrt(np.mean(dn * dn))
    e64 = np.sqrt(np.mean((np.linalg.norm(res[L.PREC_FP64][0] - d, axis=1) / scale) ** 2))
    e32 = np.sqrt(np.mean((np.linalg.norm(res[L.PREC_FP32][0] - d, axis=1) / scale) ** 2))
    assert e32 <= e64 * 1.02 + 2e-5, (e32, e64)
    assert np.all(np.isfinite(res[L.PREC_FP32][0]))


@pytest.mark.parametrize("precision", [L.PREC_FP32, L.PREC_FP64])
def test_active_walk_slices_sum_to_unsliced(precision, cuda_lib):
    ic = ics.zoom_box(log2_half=13, seed=1004, pmgrid=128)
    n = len(ic["mass"])
    act = _active(n, 0.3, 14)
    prm = ics.params_for(ic, precision=precision)
    with GravityTree(prm) as t:
        _, _, _, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        fa, fp, fn = t.gravity_tree_targets(act, oldacc)
        sa, sp, sn = np.zeros_like(fa), np.zeros_like(fp), np.zeros_like(fn)
        for s in range(3):
            t.set_target_slice(s, 3)
            a, p, ni = t.gravity_tree_targets(act, oldacc)
            sa += a
            sp += p
            sn += ni
        t.set_target_slice(0, 1)
    assert np.array_equal(sa, fa) and np.array_equal(sp, fp) and np.array_equal(sn, fn)


def test_active_walk_rejects_bad_lists(cuda_lib):
    g = load_golden("hernquist2048_iso")
    n = len(g["mass"])
    with GravityTree(_gpu_params(g["params"])) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree()
        for bad in (np.array([0, 5, 5], np.int32), np.array([1, n], np.int32), np.array([-1], np.int32)):
            with pytest.raises(L.GpuGravError) as e:
                t.gravity_tree_targets(bad)
            assert e.value.status == L.ERR_INVALID
        acc, pot, ni = t.gravity_tree_targets(np.zeros(0, np.int32))
        assert acc.shape == (0, 3)
        a1, _, _ = t.gravity_tree_targets(np.array([7], np.int32))
        af, _, _ = t.gravity_tree()
        assert np.array_equal(a1[0], af[7])
