"""Generates the golden fixtures in this directory by running the reference's own
gravity code (oracle/_ref/ref_harness_{pm,iso,ewald}, compiled from the reference tree
by oracle/ref/Makefile) on small seeded particle sets.

    python tests/golden/make_golden.py [case ...]  # needs the reference tree to build the harness

Each fixture (.npz) holds the inputs, the run parameters and the reference's
outputs: domain geometry, sorted order, 126-bit keys, top-level nodes, the full
tree (node centre/len/CoM/mass/maxsofttype/sibling/nextnode/father, particle
Nextnode/Father), and for the Barnes-Hut pass and the relative pass the
per-particle accelerations, potentials, interaction counts and OldAcc.

Node indices are stored with the library's convention Tree_MaxPart = N (the
reference run uses All.MaxPart, which domain_Decomposition enlarges).

The periodic pure-tree case (no PMGRID, Ewald-corrected) also stores the SHA-256 of the
reference's scaled Ewald correction tables (ewald_init, forcetree_ewald.c:89-254) and a sample of
their entries, which pins the table restatement without shipping the 8.8 MB tables.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from arepo_b200 import ics  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    c = {}
    # periodic TreePM box: 16^3 grid + Gaussian displacements (the 32^3 box at 1/8 size)
    g = ics.grid_box(n1=16, seed=1001, pmgrid=32)
    c["grid16_pm"] = g
    # isolated Hernquist halo
    c["hernquist2048_iso"] = ics.hernquist(2048, seed=1002)
    # two species, a dense clump, exactly coincident and nearly coincident points (MAX_TREE_LEVEL rule)
    rng = np.random.default_rng(1005)
    n = 1500
    pos = rng.uniform(0, 1, (n, 3))
    st = (rng.uniform(size=n) < 0.5).astype(np.uint8)
    pos[st == 1] = np.mod(0.5 + 0.02 * rng.normal(size=((st == 1).sum(), 3)), 1.0)
    pos[100:120] = pos[99]                  # 21 identical points: slot shifting and chained nodes
    pos[200:204] = pos[199] + 1e-13         # nearly identical
    pos[300:303] = pos[299] + [1e-9, 0, 0]  # below MAX_TREE_LEVEL resolution
    mass = np.where(st == 1, 1.0, 8.0) / n
    a = 1.25 / 64
    c["mix1500_pm"] = dict(pos=pos, mass=mass, softtype=st, softening=(0.001, 0.0003), periodic=True, box=1.0, asmth=a,
                           rcut=4.5 * a)
    # MULTIPLE_NODE_SOFTENING: heavy particles with a large softening around a clump of light ones with
    # a small softening, so that nodes whose largest softening exceeds the target's are common
    rng = np.random.default_rng(1007)
    n = 2000
    st = (np.arange(n) >= 800).astype(np.uint8)
    pos = np.where(st[:, None] == 0, np.mod(0.5 + 0.08 * rng.normal(size=(n, 3)), 1.0),
                   np.mod(0.5 + 0.03 * rng.normal(size=(n, 3)), 1.0))
    mass = np.where(st == 0, 8.0, 1.0) / n
    a = 1.25 / 64
    c["mns2000_pm"] = dict(pos=pos, mass=mass, softtype=st, softening=(0.01, 0.0008), periodic=True, box=1.0, asmth=a,
                           rcut=4.5 * a, mns=True)
    # periodic pure tree with Ewald correction: 12^3 grid + displacements in a box of size 2
    g = ics.grid_box(n1=12, seed=1006, pmgrid=32)
    c["grid12_ewald"] = dict(pos=2.0 * g["pos"], mass=g["mass"], softtype=g["softtype"],
                             softening=tuple(2.0 * e for e in g["softening"]), periodic=True, box=2.0, asmth=0.0,
                             rcut=0.0, ewald=True)
    return c


def remap(a, mp_ref, n):
    a = np.asarray(a, np.int64).copy()
    sel = a >= mp_ref
    a[sel] = a[sel] - mp_ref + n
    return a.astype(np.int32)


def main():
    if not O.build_ref():
        raise SystemExit("reference harness unavailable: the reference tree is needed to regenerate fixtures")
    want = set(sys.argv[1:])
    for name, ic in cases().items():
        if want and name not in want:
            continue
        soft = tuple(ic["softening"]) + (ic["softening"][-1],) * (2 - len(ic["softening"]))
        ewald = bool(ic.get("ewald", False))
        mns = bool(ic.get("mns", False))
        tabf = tempfile.mktemp(suffix=".bin") if ewald else None
        ref = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], ic["periodic"], box=ic["box"], asmth=ic["asmth"],
                        rcut=ic["rcut"], theta=0.7, erracc=0.0025, softening=soft, mdom=8, tnf=2.5, ewald=ewald,
                        ewald_table_out=tabf, mns=mns)
        n = len(ic["mass"])
        m = ref["tree_meta"]
        mp = m["max_part"]
        prm = dict(periodic=bool(ic["periodic"]), box=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], rcut_cells=4.5,
                   softening=list(soft), theta=0.7, erracc=0.0025, mdom=8, tnf=2.5, ewald=ewald, mns=mns)
        out = dict(
            params=np.array(json.dumps(prm)),
            pos=ic["pos"], mass=ic["mass"], softtype=ic["softtype"],
            domain=ref["domain"], order=ref["order"], key_hi=ref["key_hi"], key_lo=ref["key_lo"], top=ref["top"],
            num_nodes=np.int64(m["num_nodes"]), first_non_top=np.int64(m["first_non_top"] - mp + n),
            node_center=ref["node_center"], node_len=ref["node_len"], node_s=ref["node_s"], node_mass=ref["node_mass"],
            node_maxsoft=ref["node_maxsoft"].astype(np.uint8), node_sibling=remap(ref["node_sibling"], mp, n),
            node_nextnode=remap(ref["node_nextnode"], mp, n), node_father=remap(ref["node_father"], mp, n),
            p_next=remap(ref["p_next"], mp, n), p_father=remap(ref["p_father"], mp, n),
        )
        if mns:
            out["node_mpt"] = ref["node_mpt"]
        if ewald:
            raw = open(tabf, "rb").read()
            os.remove(tabf)
            sz = int(np.frombuffer(raw[:8], np.int64)[0])
            tab = np.frombuffer(raw[16:], np.float64).reshape(4, sz)
            out["ewald_fac_intp"] = np.frombuffer(raw[8:16], np.float64)[0]
            out["ewald_sha256"] = np.array(hashlib.sha256(tab.tobytes()).hexdigest())
            idx = np.random.default_rng(7).choice(sz, 64, replace=False)
            out["ewald_sample_idx"] = idx
            out["ewald_sample"] = tab[:, idx]
        for ps in range(2):
            for k in ("acc", "pot", "ninter", "oldacc"):
                out[f"{k}{ps}"] = ref[f"{k}{ps}"]
            assert np.array_equal(ref[f"gacc{ps}"], ref[f"acc{ps}"]), "gravity_tree and force_treeevaluate disagree"
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: N={n} nodes={m['num_nodes']} NTopnodes={m['ntopnodes']} "
              f"ia/part={out['ninter1'].mean():.1f} size={os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
