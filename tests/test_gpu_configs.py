"""The benchmark configurations at their stated sizes and parameters.

C1  32^3 grid box (seed 1001, sigma 0.2 spacing, PMGRID 64, softening 1/40 spacing, BH 0.7 then
    relative 0.0025): FP64 bit-exact against the C oracle's whole pipeline and, where the reference
    harness is built, against the reference's own gravity_tree on the same particles.
C2  2^20 Hernquist halo (seed 1002, isolated, softening 0.01): keys, order, top tree and every node
    bit-exact; both passes bit-exact on every 256th target (the C oracle, and the reference harness
    where it is built); FP32 against the FP64 direct sum on 4096 random targets (seed 2002).
C3  256^3 Zel'dovich box (seed 1003, PMGRID 512, softening 1/30 spacing): FP32 and FP64 walks against
    the FP64 direct sum on 8192 random targets (seed 2003).

Accuracy is stated as e_i = |a_i - a_i^ref| / |a_i^ref| with its RMS and 99th percentile; the FP32 walk
must be no less accurate than the FP64 parity walk (the reference's decisions) on the same targets."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from oracle import oracle as O
from test_gpu_parity import assert_tree_equal, top_equal

pytestmark = pytest.mark.gpu


def _rel(acc, ref):
    e = np.linalg.norm(acc - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
    return float(np.sqrt(np.mean(e * e))), float(np.percentile(e, 99))


def _oracle_tree_dict(o):
    return dict(num_nodes=o["num_nodes"], first_non_top=o["first_non_top"], node_center=o["center"], node_len=o["len"],
                node_s=o["s"], node_mass=o["mass"], node_maxsoft=o["maxsoft"], node_sibling=o["sibling"],
                node_nextnode=o["nextnode"], node_father=o["father"], p_next=o["p_next"], p_father=o["p_father"])


def test_c1_grid_box_bitexact(cuda_lib):
    ic = ics.grid_box(n1=32, sigma_cells=0.2, seed=1001, pmgrid=64, soft_frac=1 / 40)
    eps = ic["softening"][0]
    soft = (eps, eps)  # two softening types (the harness build's NSOFTTYPES), every particle of type 0
    op = O.make_params(True, box=1.0, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft)
    ref = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], op)
    prm = L.make_params(True, box_size=1.0, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft)
    with GravityTree(prm) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        order = t.order()
        tr = t.export_tree()
    assert np.array_equal(order, ref["perm"])
    assert_tree_equal(tr, _oracle_tree_dict(ref["tree"]))
    assert np.array_equal(oldacc[order], ref["oldacc0"])
    assert np.array_equal(acc[order], ref["acc1"]) and np.array_equal(pot[order], ref["pot1"])
    assert np.array_equal(ni[order], ref["ninter1"])
    if O.ref_available():
        r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft,
                      dump=0, gt=1)
        assert np.array_equal(order, r["order"])
        assert np.array_equal(acc[order], r["acc1"])  # the reference's force_treeevaluate per target
        assert np.array_equal(acc[order], r["gacc1"])  # the reference's gravity_tree, relative pass


def test_c2_hernquist_2e20(cuda_lib):
    ic = ics.hernquist(1 << 20, seed=1002)
    n = len(ic["mass"])
    soft = (ic["softening"][0], ic["softening"][0])
    op = O.make_params(False, softening=soft, theta=0.7, erracc=0.0025)
    pos = O.wrap(ic["pos"], op)
    dom = O.extent(pos, op)
    hi, lo, ip = O.keys(pos, op, dom)
    perm = O.sort(hi, lo)
    top = O.toptree(hi[perm], lo[perm], op)
    tree = O.build(pos[perm], ic["mass"][perm], ic["softtype"][perm], ip[perm], op, dom, top)
    tg = np.arange(0, n, 256)  # sorted positions
    ps, ms, ss = pos[perm], ic["mass"][perm], ic["softtype"][perm]
    a0, _, _ = O.walk(tree, ps, ms, ss, np.zeros(n, np.float32), op, targets=tg)
    old_s = np.zeros(n, np.float32)
    old_s[tg] = np.sqrt(np.sum(a0 * a0, axis=1)).astype(np.float32)  # gravity_force_finalize without PM
    op.theta = 0.0
    a1, p1, n1 = O.walk(tree, ps, ms, ss, old_s, op, targets=tg)

    prm = L.make_params(False, softening=soft, err_tol_theta=0.7, err_tol_force_acc=0.0025)
    with GravityTree(prm) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        order = t.order()
        kh, kl = t.keys()
        assert top_equal(t.topnodes(), top)
        assert_tree_equal(t.export_tree(), _oracle_tree_dict(tree))
    assert np.array_equal(order, perm)
    assert np.array_equal(kh, hi[perm]) and np.array_equal(kl, lo[perm])
    assert np.array_equal(oldacc[order][tg], old_s[tg])
    assert np.array_equal(acc[order][tg], a1) and np.array_equal(pot[order][tg], p1) and np.array_equal(ni[order][tg], n1)
    if O.ref_available():
        r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], False, softening=soft, stride=256, dump=0, gt=0)
        assert np.array_equal(r["order"], order)
        assert np.array_equal(r["acc1"][tg], a1) and np.array_equal(r["ninter1"][tg], n1)

    # FP32 walk against the FP64 direct sum on 4096 random targets
    rt = np.sort(np.random.default_rng(2002).choice(n, 4096, replace=False))
    with GravityTree(L.make_params(False, softening=soft, err_tol_theta=0.7, err_tol_force_acc=0.0025,
                                   precision=L.PREC_FP32)) as t:
        a32, _, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        d, _ = t.direct(rt)
    rms64, p64 = _rel(acc[rt], d)
    rms32, p32 = _rel(a32[rt], d)
    print(f"C2 vs FP64 direct sum: FP64 walk rms {rms64:.3e} p99 {p64:.3e}; FP32 walk rms {rms32:.3e} p99 {p32:.3e}")
    assert rms32 <= rms64 * 1.02 + 2e-5, (rms32, rms64)


def test_c3_zeldovich_256(cuda_lib):
    ic = ics.zeldovich_box(n1=256, seed=1003, pmgrid=512, rms_cells=0.5, soft_frac=1 / 30)
    n = len(ic["mass"])
    rt = np.sort(np.random.default_rng(2003).choice(n, 8192, replace=False))
    res = {}
    for prec in (L.PREC_FP64, L.PREC_FP32):
        with GravityTree(ics.params_for(ic, precision=prec)) as t:
            acc, _, ni, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
            res[prec] = (acc[rt], int(ni.sum()))
            if prec == L.PREC_FP64:
                d_cut, _ = t.direct(rt, cut=True)
    rms64, p64 = _rel(res[L.PREC_FP64][0], d_cut)
    rms32, p32 = _rel(res[L.PREC_FP32][0], d_cut)
    print(f"C3 vs FP64 direct sum (r < Rcut): FP64 walk rms {rms64:.3e} p99 {p64:.3e} ({res[L.PREC_FP64][1] / n:.0f} ia/p); "
          f"FP32 walk rms {rms32:.3e} p99 {p32:.3e} ({res[L.PREC_FP32][1] / n:.0f} ia/p)")
    assert rms32 <= rms64 * 1.02 + 2e-5, (rms32, rms64)
    assert np.all(np.isfinite(res[L.PREC_FP32][0]))
