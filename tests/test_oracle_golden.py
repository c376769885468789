"""The C oracle against golden fixtures made by the reference's own compiled code
(tests/golden/make_golden.py).  Everything is compared bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from oracle import oracle as O


def oracle_params(g):
    p = g["params"]
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


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference(name):
    g = load_golden(name)
    prm = oracle_params(g)
    out = O.pipeline(g["pos"], g["mass"], g["softtype"], prm, top=g["top"])
    d = out["domain"]
    assert np.array_equal(np.array(list(d.corner) + list(d.center) + [d.len, d.inverse_len, d.big_fac]), g["domain"][:9])
    assert np.array_equal(out["perm"], g["order"])
    assert np.array_equal(out["key_hi"][out["perm"]], g["key_hi"])
    assert np.array_equal(out["key_lo"][out["perm"]], g["key_lo"])
    t = out["tree"]
    assert t["num_nodes"] == int(g["num_nodes"])
    assert t["first_non_top"] == int(g["first_non_top"])
    for k_or, k_g in (("center", "node_center"), ("len", "node_len"), ("s", "node_s"), ("mass", "node_mass"),
                      ("maxsoft", "node_maxsoft"), ("sibling", "node_sibling"), ("nextnode", "node_nextnode"),
                      ("father", "node_father"), ("p_next", "p_next"), ("p_father", "p_father")):
        assert np.array_equal(t[k_or], g[k_g]), k_or
    if "node_mpt" in g:
        assert np.array_equal(O.mass_per_type(t, out["mass_sorted"], out["st_sorted"], prm), g["node_mpt"])
    for ps in range(2):
        assert np.array_equal(out[f"acc{ps}"], g[f"acc{ps}"])
        assert np.array_equal(out[f"pot{ps}"], g[f"pot{ps}"])
        assert np.array_equal(out[f"ninter{ps}"], g[f"ninter{ps}"])
        assert np.array_equal(out[f"oldacc{ps}"], g[f"oldacc{ps}"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_top_tree_matches_reference(name):
    """Count-based top tree of the oracle equals the reference's domain_determineTopTree here."""
    g = load_golden(name)
    prm = oracle_params(g)
    pos = O.wrap(g["pos"], prm)
    dom = O.extent(pos, prm)
    hi, lo, ip = O.keys(pos, prm, dom)
    perm = O.sort(hi, lo)
    top = O.toptree(hi[perm], lo[perm], prm)
    assert top_equal(top, g["top"])
    # MortonToPeanoSubnode recomputed from StartKey/Size (domain.c:246-272)
    t2 = np.ascontiguousarray(g["top"].copy())
    t2["morton_to_peano"] = 0
    O.lib().or_topnode_m2p(len(t2), t2.ctypes.data_as(O.C.c_void_p))
    assert np.array_equal(t2["morton_to_peano"], g["top"]["morton_to_peano"])


def test_ewald_tables_match_reference():
    """The restated Ewald correction tables (ewald_init, forcetree_ewald.c:154-251) scaled to the
    fixture's box: the same bytes as the reference's (SHA-256 and sampled entries)."""
    import hashlib

    g = load_golden("grid12_ewald")
    box = g["params"]["box"]
    t = O.ewald_table()
    scaled = np.stack([t[0] / (box * box), t[1] / (box * box), t[2] / (box * box), t[3] / box])
    assert np.array_equal(scaled[:, g["ewald_sample_idx"]], g["ewald_sample"])
    assert hashlib.sha256(np.ascontiguousarray(scaled).tobytes()).hexdigest() == str(g["ewald_sha256"])
    assert float(g["ewald_fac_intp"]) == 2 * O.EWALD_EN / box


def test_shortrange_table_matches_reference_formula():
    f, p = O.shortrange_table(4.5)
    assert f[0] == 0.0 and p[0] == np.float32(-1.0)
    assert np.all(np.diff(p) > 0)  # -erfc(u) increases
    assert f.dtype == np.float32 and len(f) == O.NTAB + 1


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_walk_close_to_direct_sum(name):
    """Sanity: tree accelerations approximate the FP64 direct sum (relative criterion).
    Errors are normalised by the RMS force of the sample: in the low-density part of a
    TreePM box the short-range force itself is close to zero."""
    g = load_golden(name)
    prm = oracle_params(g)
    tg = np.arange(0, len(g["mass"]), 7)
    acc_d, _ = O.direct(O.wrap(g["pos"], prm), g["mass"], g["softtype"], prm, tg)
    inv = np.empty_like(g["order"])
    inv[g["order"]] = np.arange(len(inv))
    acc_t = g["acc1"][inv[tg]]
    scale = np.sqrt(np.mean(np.sum(acc_d * acc_d, axis=1)))
    err = np.linalg.norm(acc_t - acc_d, axis=1) / scale
    assert np.sqrt(np.mean(err ** 2)) < 2e-2


def test_oracle_minimum_opening_angle_matches_reference_build():
    """The oracle's ACTIVATE_MINIMUM_OPENING_ANGLE flag against a harness build of the reference with that
    option (oracle/ref/config_pm_mina.h), both passes bit for bit; skipped where the harness is not built."""
    import os

    if not os.path.exists(os.path.join(O.REF_DIR, "ref_harness_pm_mina")):
        pytest.skip("reference harness with ACTIVATE_MINIMUM_OPENING_ANGLE not built")
    from arepo_b200 import ics

    ic = ics.zoom_box(log2_half=12, seed=52, pmgrid=64)
    soft = tuple(ic["softening"])
    prm = O.make_params(True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft, minangle=True)
    out = O.pipeline(ic["pos"], ic["mass"], ic["softtype"], prm)
    r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft, dump=0,
                  gt=0, minangle=True)
    assert np.array_equal(out["perm"], r["order"])
    for ps in (0, 1):
        assert np.array_equal(out[f"acc{ps}"], r[f"acc{ps}"]) and np.array_equal(out[f"ninter{ps}"], r[f"ninter{ps}"])
