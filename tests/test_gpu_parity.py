"""Parity of the CUDA path (through the C ABI) with the reference.

Golden fixtures were produced by the reference's own compiled code; the live
checks compare with the C oracle, which the CPU tests pin bit-for-bit to the
same fixtures.  The FP64 path must reproduce keys, order, top tree, tree
(reference node numbering) and per-particle accelerations, potentials and
interaction counts bit for bit."""
import os

import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from conftest import GOLDEN_CASES, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_params(p, precision=L.PREC_FP64):
    return L.make_params(periodic=p["periodic"], box_size=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                         rcut_cells=p["rcut_cells"], softening=tuple(p["softening"]), err_tol_theta=p["theta"],
                         err_tol_force_acc=p["erracc"], top_node_factor=p["tnf"], multiple_domains=p["mdom"],
                         precision=precision, multiple_node_softening=p.get("mns", False))


def oracle_params(p):
    return O.make_params(p["periodic"], box=p["box"], asmth=p["asmth"], rcut=p["rcut"], rcut_cells=p["rcut_cells"],
                         theta=p["theta"], erracc=p["erracc"], softening=tuple(p["softening"]), mdom=p["mdom"], tnf=p["tnf"],
                         mns=p.get("mns", False))


def top_equal(a, b):
    if len(a) != len(b):
        return False
    for f in ("start_hi", "start_lo", "size_hi", "size_lo", "daughter", "morton_to_peano"):
        if not np.array_equal(a[f], b[f]):
            return False
    leaf = a["daughter"] < 0
    return np.array_equal(a["leaf"][leaf], b["leaf"][leaf])


def assert_tree_equal(t, g):
    assert t["num_nodes"] == int(g["num_nodes"])
    assert t["first_non_top"] == int(g["first_non_top"])
    for k, kg in (("center", "node_center"), ("len", "node_len"), ("s", "node_s"), ("mass", "node_mass"),
                  ("maxsoft", "node_maxsoft"), ("sibling", "node_sibling"), ("nextnode", "node_nextnode"),
                  ("father", "node_father"), ("p_next", "p_next"), ("p_father", "p_father")):
        a, b = np.asarray(t[k]), np.asarray(g[kg])
        assert a.shape == b.shape, k
        bad = np.flatnonzero(np.any((a != b).reshape(len(a), -1), axis=1))
        assert len(bad) == 0, f"{k}: {len(bad)} entries differ, first {bad[:5]}"


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_domain_keys_order_bitexact(name, cuda_lib):
    g = load_golden(name)
    with GravityTree(gpu_params(g["params"])) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        d = t.domain()
        assert np.array_equal(np.array(list(d.corner) + list(d.center) + [d.len, d.inverse_len, d.big_fac]), g["domain"][:9])
        assert np.array_equal(t.order(), g["order"])
        hi, lo = t.keys()
        assert np.array_equal(hi, g["key_hi"]) and np.array_equal(lo, g["key_lo"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_tree_bitexact_with_reference_topnodes(name, cuda_lib):
    g = load_golden(name)
    with GravityTree(gpu_params(g["params"])) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree(topnodes=g["top"])
        assert_tree_equal(t.export_tree(), g)
        if "node_mpt" in g:  # MULTIPLE_NODE_SOFTENING: ExtNodes[].mass_per_type
            assert np.array_equal(t.mass_per_type(), g["node_mpt"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_library_top_tree_equals_reference(name, cuda_lib):
    g = load_golden(name)
    with GravityTree(gpu_params(g["params"])) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree()
        assert top_equal(t.topnodes(), g["top"])
        assert_tree_equal(t.export_tree(), g)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_walk_bitexact_both_passes(name, cuda_lib):
    g = load_golden(name)
    order = g["order"]
    prm = gpu_params(g["params"])
    with GravityTree(prm) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree(topnodes=g["top"])
        acc, pot, ni = t.gravity_tree()
        assert np.array_equal(acc[order], g["acc0"])
        assert np.array_equal(pot[order], g["pot0"])
        assert np.array_equal(ni[order], g["ninter0"])
        # relative criterion with the reference's OldAcc (float)
        oldacc = np.empty(len(order), np.float32)
        oldacc[order] = g["oldacc0"]
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        acc, pot, ni = t.gravity_tree(oldacc)
        assert np.array_equal(acc[order], g["acc1"])
        assert np.array_equal(pot[order], g["pot1"])
        assert np.array_equal(ni[order], g["ninter1"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_compute_grav_accelerations_sequence(name, cuda_lib):
    """BH pass, OldAcc, relative pass through the reference-shaped driver."""
    g = load_golden(name)
    order = g["order"]
    with GravityTree(gpu_params(g["params"])) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(g["pos"], g["mass"], g["softtype"], topnodes=g["top"])
    assert np.array_equal(oldacc[order], g["oldacc0"])
    assert np.array_equal(acc[order], g["acc1"])
    assert np.array_equal(ni[order], g["ninter1"])


def _live_case(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "grid":
        n1 = int(round(n ** (1 / 3)))
        return ics.grid_box(n1=n1, seed=seed, pmgrid=2 * n1)
    if kind == "hernquist":
        return ics.hernquist(n, seed=seed)
    if kind == "zoom":
        k = int(np.log2(n // 2))
        return ics.zoom_box(log2_half=k, seed=seed, pmgrid=64)
    if kind == "coincident":
        pos = rng.uniform(0, 1, (n, 3))
        for b in range(40):
            i = rng.integers(0, n - 200)
            pos[i + 1:i + 1 + int(rng.integers(2, 60))] = pos[i]
        a = 1.25 / 32
        return dict(pos=pos, mass=rng.uniform(0.5, 1.5, n) / n, softtype=(rng.uniform(size=n) < 0.3).astype(np.uint8),
                    softening=(0.002, 0.004), periodic=True, box=1.0, asmth=a, rcut=4.5 * a)
    raise ValueError(kind)


@pytest.mark.parametrize("kind,n,seed", [("grid", 32768, 7), ("hernquist", 40000, 8), ("zoom", 32768, 9),
                                         ("coincident", 20000, 10)])
def test_live_cases_bitexact_vs_oracle(kind, n, seed, cuda_lib):
    ic = _live_case(kind, n, seed)
    soft = tuple(ic["softening"])
    p = dict(periodic=ic["periodic"], box=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], rcut_cells=4.5, softening=soft,
             theta=0.7, erracc=0.0025, mdom=8, tnf=2.5)
    ref = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], oracle_params(p))
    order = ref["perm"]
    with GravityTree(gpu_params(p)) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        assert np.array_equal(t.order(), order)
        assert top_equal(t.topnodes(), ref["top"])
        tr = t.export_tree()
        info = t.tree_info()
    o = ref["tree"]
    g = dict(num_nodes=o["num_nodes"], first_non_top=o["first_non_top"], node_center=o["center"], node_len=o["len"],
             node_s=o["s"], node_mass=o["mass"], node_maxsoft=o["maxsoft"], node_sibling=o["sibling"],
             node_nextnode=o["nextnode"], node_father=o["father"], p_next=o["p_next"], p_father=o["p_father"])
    assert_tree_equal(tr, g)
    assert np.array_equal(oldacc[order], ref["oldacc0"])
    assert np.array_equal(acc[order], ref["acc1"])
    assert np.array_equal(pot[order], ref["pot1"])
    assert np.array_equal(ni[order], ref["ninter1"])
    if kind == "coincident":
        assert info.coincident_cells > 0


def test_direct_sum_matches_oracle(cuda_lib):
    g = load_golden("grid16_pm")
    p = g["params"]
    tg = np.arange(0, len(g["mass"]), 13)
    with GravityTree(gpu_params(p)) as t:
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        acc, pot = t.direct(tg)
    acc_o, pot_o = O.direct(O.wrap(g["pos"], oracle_params(p)), g["mass"], g["softtype"], oracle_params(p), tg)
    # CUDA's and glibc's erfc/exp differ by a few ulp; the summation order differs
    scale = np.max(np.abs(acc_o))
    assert np.max(np.abs(acc - acc_o)) < 1e-11 * scale
    assert np.max(np.abs(pot - pot_o)) < 1e-11 * np.max(np.abs(pot_o))


def test_error_codes(cuda_lib):
    g = load_golden("hernquist2048_iso")
    prm = gpu_params(g["params"])
    with GravityTree(prm) as t:
        with pytest.raises(L.GpuGravError) as e:
            t.gravity_tree()
        assert e.value.status == L.ERR_STATE
        # a domain that does not contain every particle -> -3 (forcetree.c:411-430)
        d = L.Domain()
        for j in range(3):
            d.corner[j] = -1.0
            d.center[j] = 0.0
        d.len, d.inverse_len, d.big_fac = 2.0, 0.5, 2.0 / 2 ** 52
        with pytest.raises(L.GpuGravError) as e:
            t.domain_decomposition(g["pos"], g["mass"], g["softtype"], domain=d)
        assert e.value.status == L.ERR_OUT_OF_BOX
        bad = g["pos"].copy()
        bad[5, 1] = np.nan
        with pytest.raises(L.GpuGravError) as e:
            t.domain_decomposition(bad, g["mass"], g["softtype"])
        assert e.value.status == L.ERR_INVALID
        st = g["softtype"].copy()
        st[3] = 7
        with pytest.raises(L.GpuGravError) as e:
            t.domain_decomposition(g["pos"], g["mass"], st)
        assert e.value.status == L.ERR_INVALID
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        top = g["top"].copy()
        top["daughter"][0] = 10 ** 6
        with pytest.raises(L.GpuGravError) as e:
            t.construct_forcetree(topnodes=top)
        assert e.value.status == L.ERR_TOPNODES
        # the context stays usable after errors
        t.domain_decomposition(g["pos"], g["mass"], g["softtype"])
        t.construct_forcetree(topnodes=g["top"])
        acc, _, _ = t.gravity_tree()
        assert np.array_equal(acc[g["order"]], g["acc0"])


def test_minimum_opening_angle_bitexact(cuda_lib):
    """ACTIVATE_MINIMUM_OPENING_ANGLE (GPUGRAV_FLAG_MINIMUM_OPENING_ANGLE): both passes bit-exact with
    the C oracle, which is pinned to a harness build of the reference with that option where it is built;
    the FP32 walk with the flag stays no less accurate than the FP64 walk."""
    ic = _live_case("zoom", 32768, 51)
    soft = tuple(ic["softening"])
    p = dict(periodic=True, box=1.0, asmth=ic["asmth"], rcut=ic["rcut"], rcut_cells=4.5, softening=soft, theta=0.7,
             erracc=0.0025, mdom=8, tnf=2.5)
    op = oracle_params(p)
    op.flags |= 2
    ref = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], op)
    order = ref["perm"]
    prm = gpu_params(p)
    prm.flags |= L.FLAG_MINIMUM_OPENING_ANGLE
    with GravityTree(prm) as t:
        acc, pot, ni, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
    assert np.array_equal(oldacc[order], ref["oldacc0"])
    assert np.array_equal(acc[order], ref["acc1"]) and np.array_equal(ni[order], ref["ninter1"])
    plain = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], oracle_params(p))
    assert ref["ninter1"].sum() < plain["ninter1"].sum()  # the option opens fewer nodes
    if O.ref_available() and os.path.exists(os.path.join(O.REF_DIR, "ref_harness_pm_mina")):
        r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft,
                      dump=0, gt=0, minangle=True)
        assert np.array_equal(r["acc1"], ref["acc1"]) and np.array_equal(r["ninter1"], ref["ninter1"])
