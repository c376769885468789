"""TEST INFRASTRUCTURE ONLY -- Python access to the oracles.

Two oracles live under ``oracle/``:

* ``gpugrav_oracle.c``: a plain-C restatement of the reference's short-range
  tree-gravity path (keys, sort, top tree, tree build, moments, walk, direct
  summation), built into ``oracle/_build/liboracle.so``;
* ``ref/``: a recipe that compiles the reference's own sources into
  ``oracle/_ref/ref_harness_{pm,iso}`` (only where the reference tree is present).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the library under ``arepo_b200/`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
SRC_PATH = os.path.join(HERE, "gpugrav_oracle.c")

NTAB = 127
MAX_SOFT = 16

TOPNODE_DTYPE = np.dtype(
    [
        ("start_hi", "<u8"),
        ("start_lo", "<u8"),
        ("size_hi", "<u8"),
        ("size_lo", "<u8"),
        ("daughter", "<i4"),
        ("leaf", "<i4"),
        ("morton_to_peano", "u1", (8,)),
    ]
)
assert TOPNODE_DTYPE.itemsize == 48


class OrParams(C.Structure):
    _fields_ = [
        ("periodic", C.c_int),
        ("nsoft", C.c_int),
        ("box", C.c_double),
        ("asmth", C.c_double),
        ("rcut", C.c_double),
        ("rcut_cells", C.c_double),
        ("theta", C.c_double),
        ("erracc", C.c_double),
        ("tnf", C.c_double),
        ("mdom", C.c_int),
        ("flags", C.c_int),  # bit 0: MULTIPLE_NODE_SOFTENING, bit 1: ACTIVATE_MINIMUM_OPENING_ANGLE
        ("soft", C.c_double * MAX_SOFT),
    ]


class OrDomain(C.Structure):
    _fields_ = [
        ("corner", C.c_double * 3),
        ("center", C.c_double * 3),
        ("len", C.c_double),
        ("inverse_len", C.c_double),
        ("big_fac", C.c_double),
    ]


def build_oracle(force: bool = False) -> str:
    """Compile the C restatement (plain -O2, no FMA contraction on x86-64)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC_PATH):
        subprocess.check_call(
            ["gcc", "-std=gnu11", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", LIB_PATH, SRC_PATH, "-lm"]
        )
    return LIB_PATH


def build_ref(ref_root: str | None = None) -> bool:
    """Compile the reference harness from the reference tree at ref_root (default: the AREPO_REFERENCE
    environment variable) when that tree is present; returns availability."""
    ref_root = ref_root or os.environ.get("AREPO_REFERENCE", "")
    if ref_root and os.path.isdir(os.path.join(ref_root, "src", "gravity")):
        subprocess.check_call(
            ["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), f"REF={ref_root}", f"OUT={REF_DIR}"]
        )
        # the builds that call the library through its C binding, once the library exists
        if os.path.exists(os.path.join(os.path.dirname(HERE), "arepo_b200", "libarepo_gpugrav.so")):
            subprocess.check_call(
                ["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), f"REF={ref_root}", f"OUT={REF_DIR}", "gpu"]
            )
    return ref_available()


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"ref_harness_{c}")) for c in ("pm", "iso"))


def ref_gpu_available() -> bool:
    """the harness builds whose gravity step calls the library through its C binding"""
    return all(os.path.exists(os.path.join(REF_DIR, f"ref_harness_{c}_gpu")) for c in ("pm", "iso"))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_oracle())
        p = C.c_void_p
        i64 = C.c_int64
        _lib.or_extent.argtypes = [i64, p, p, p]
        _lib.or_keys.argtypes = [i64, p, p, p, p, p, p]
        _lib.or_sort.argtypes = [i64, p, p, p]
        _lib.or_toptree.argtypes = [i64, p, p, p, p, C.c_int]
        _lib.or_toptree.restype = C.c_int
        _lib.or_topnode_m2p.argtypes = [C.c_int, p]
        _lib.or_build.argtypes = [i64, p, p, p, p, p, p, p, C.c_int, i64, i64] + [p] * 11 + [p]
        _lib.or_build.restype = i64
        _lib.or_shortrange_table.argtypes = [C.c_double, p, p]
        _lib.or_walk.argtypes = [i64, p, p, p, p, p, p, p, p, i64, i64, p, p, p, p, p, p, p, p, p, p, p, p]
        _lib.or_mass_per_type.argtypes = [i64, p, i64, p, p, C.c_int, p]
        _lib.or_mass_per_type.restype = C.c_int
        _lib.or_direct.argtypes = [i64, p, i64, p, p, p, p, p, p]
        _lib.or_gravity_direct.argtypes = [i64, p, p, p, p, p, p]
        _lib.or_timestep_gravity.argtypes = [i64, p, p, p, p, p, p, p, p, p, p]
        _lib.or_timestep_gravity.restype = C.c_int
        _lib.or_ewald_table.argtypes = [p, p, p, p]
        _lib.or_set_ewald_table.argtypes = [C.c_double, p, p, p, p]
    return _lib


EWALD_EN = 64
_ewald_unscaled = None
_ewald_scaled = {}


def ewald_table():
    """The unscaled Ewald correction tables of ewald_init (forcetree_ewald.c:154-185), computed by
    the C restatement (about 30 CPU-seconds, OpenMP) and cached in oracle/_build."""
    global _ewald_unscaled
    if _ewald_unscaled is None:
        f = os.path.join(BUILD_DIR, f"ewald_table_{EWALD_EN}.npy")
        if os.path.exists(f):
            _ewald_unscaled = np.load(f)
        else:
            m = (EWALD_EN + 1) ** 3
            t = np.zeros((4, m))
            lib().or_ewald_table(_ptr(t[0]), _ptr(t[1]), _ptr(t[2]), _ptr(t[3]))
            os.makedirs(BUILD_DIR, exist_ok=True)
            np.save(f, t)
            _ewald_unscaled = t
    return _ewald_unscaled


def use_ewald(prm):
    """Install the tables scaled to prm.box (fcorr / L^2, potcorr / L, forcetree_ewald.c:239-251) for
    the walk and direct sum of a periodic pure-tree parameter set (periodic, asmth == 0)."""
    if not (prm.periodic and prm.asmth == 0):
        return
    box = float(prm.box)
    if box not in _ewald_scaled:
        t = ewald_table()
        _ewald_scaled[box] = np.ascontiguousarray(np.stack([t[0] / (box * box), t[1] / (box * box), t[2] / (box * box),
                                                            t[3] / box]))
    s = _ewald_scaled[box]
    lib().or_set_ewald_table(box, _ptr(s[0]), _ptr(s[1]), _ptr(s[2]), _ptr(s[3]))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def make_params(
    periodic: bool,
    box: float = 1.0,
    asmth: float = 0.0,
    rcut: float = 0.0,
    rcut_cells: float = 4.5,
    theta: float = 0.7,
    erracc: float = 0.0025,
    softening=(0.01, 0.01),
    mdom: int = 8,
    tnf: float = 2.5,
    mns: bool = False,
    minangle: bool = False,
) -> OrParams:
    """softening: Plummer-equivalent epsilon per type; ForceSoftening = 2.8*eps (set_softenings,
    src/gravity/grav_softening.c:92-95) with a trailing zero entry."""
    p = OrParams()
    p.periodic = 1 if periodic else 0
    p.nsoft = len(softening)
    p.box = box
    p.asmth = asmth
    p.rcut = rcut
    p.rcut_cells = rcut_cells
    p.theta = theta
    p.erracc = erracc
    p.tnf = tnf
    p.mdom = mdom
    p.flags = (1 if mns else 0) | (2 if minangle else 0)
    for i, e in enumerate(softening):
        p.soft[i] = 2.8 * e
    p.soft[len(softening)] = 0.0
    return p


def extent(pos: np.ndarray, prm: OrParams) -> OrDomain:
    d = OrDomain()
    pos = np.ascontiguousarray(pos, np.float64)
    lib().or_extent(len(pos), _ptr(pos), C.byref(prm), C.byref(d))
    return d


def keys(pos, prm, dom):
    pos = np.ascontiguousarray(pos, np.float64)
    n = len(pos)
    hi = np.zeros(n, np.uint64)
    lo = np.zeros(n, np.uint64)
    ip = np.zeros((n, 3), np.uint64)
    lib().or_keys(n, _ptr(pos), C.byref(prm), C.byref(dom), _ptr(hi), _ptr(lo), _ptr(ip))
    return hi, lo, ip


def sort(hi, lo):
    n = len(hi)
    perm = np.zeros(n, np.int64)
    lib().or_sort(n, _ptr(np.ascontiguousarray(hi)), _ptr(np.ascontiguousarray(lo)), _ptr(perm))
    return perm


def toptree(hi_sorted, lo_sorted, prm, max_top: int = 4096):
    out = np.zeros(max_top, TOPNODE_DTYPE)
    nt = lib().or_toptree(len(hi_sorted), _ptr(np.ascontiguousarray(hi_sorted)), _ptr(np.ascontiguousarray(lo_sorted)),
                          C.byref(prm), _ptr(out), max_top)
    if nt < 0:
        raise RuntimeError("top tree construction failed")
    return out[:nt].copy()


def wrap(pos, prm):
    pos = np.array(pos, np.float64)
    if prm.periodic:
        pos = np.where(pos < 0, pos + prm.box, pos)
        pos = np.where(pos >= prm.box, pos - prm.box, pos)
    return pos


def build(pos_sorted, mass_sorted, st_sorted, ip_sorted, prm, dom, top, max_part=None, max_nodes=None):
    n = len(mass_sorted)
    max_part = n if max_part is None else max_part
    max_nodes = max(8 * n + 8 * len(top) + 64, 1024) if max_nodes is None else max_nodes
    arrs = dict(
        suns=np.zeros((max_nodes, 8), np.int32),
        center=np.zeros((max_nodes, 3)),
        len=np.zeros(max_nodes),
        s=np.zeros((max_nodes, 3)),
        mass=np.zeros(max_nodes),
        sibling=np.zeros(max_nodes, np.int32),
        nextnode=np.zeros(max_nodes, np.int32),
        father=np.zeros(max_nodes, np.int32),
        maxsoft=np.zeros(max_nodes, np.uint8),
        p_next=np.zeros(n, np.int32),
        p_father=np.zeros(n, np.int32),
    )
    fnt = C.c_int64(0)
    pos_sorted = np.ascontiguousarray(pos_sorted, np.float64)
    mass_sorted = np.ascontiguousarray(mass_sorted, np.float64)
    st_sorted = np.ascontiguousarray(st_sorted, np.uint8)
    ip_sorted = np.ascontiguousarray(ip_sorted, np.uint64)
    top = np.ascontiguousarray(top, TOPNODE_DTYPE)
    nn = lib().or_build(
        n, _ptr(pos_sorted), _ptr(mass_sorted), _ptr(st_sorted), _ptr(ip_sorted), C.byref(prm), C.byref(dom), _ptr(top),
        len(top), max_part, max_nodes,
        *[_ptr(arrs[k]) for k in ("suns", "center", "len", "s", "mass", "sibling", "nextnode", "father", "maxsoft",
                                   "p_next", "p_father")],
        C.byref(fnt),
    )
    if nn < 0:
        raise RuntimeError(f"tree build failed ({nn})")
    tree = {k: (v[:nn].copy() if k not in ("p_next", "p_father") else v) for k, v in arrs.items()}
    tree.update(num_nodes=int(nn), max_part=int(max_part), first_non_top=int(fnt.value))
    return tree


def walk(tree, pos_sorted, mass_sorted, st_sorted, oldacc_sorted, prm, targets=None):
    use_ewald(prm)
    n = len(mass_sorted)
    tg = None if targets is None else np.ascontiguousarray(targets, np.int64)
    nt = n if targets is None else len(tg)
    acc = np.zeros((nt, 3))
    pot = np.zeros(nt)
    ninter = np.zeros(nt, np.int32)
    pos_sorted = np.ascontiguousarray(pos_sorted, np.float64)
    mass_sorted = np.ascontiguousarray(mass_sorted, np.float64)
    st_sorted = np.ascontiguousarray(st_sorted, np.uint8)
    oldacc_sorted = np.ascontiguousarray(oldacc_sorted, np.float32)
    mpt = None
    if prm.flags & 1:
        mpt = mass_per_type(tree, mass_sorted, st_sorted, prm)
    lib().or_walk(
        nt, _ptr(tg), _ptr(pos_sorted), _ptr(oldacc_sorted), _ptr(st_sorted), _ptr(pos_sorted), _ptr(mass_sorted),
        _ptr(st_sorted), _ptr(tree["p_next"]), tree["max_part"], tree["num_nodes"], _ptr(tree["center"]),
        _ptr(tree["len"]), _ptr(tree["s"]), _ptr(tree["mass"]), _ptr(tree["sibling"]), _ptr(tree["nextnode"]),
        _ptr(tree["maxsoft"]), C.byref(prm), _ptr(acc), _ptr(pot), _ptr(ninter), _ptr(mpt),
    )
    return acc, pot, ninter


def mass_per_type(tree, mass_sorted, st_sorted, prm):
    """Per-node masses per softening type (MULTIPLE_NODE_SOFTENING's ExtNodes[].mass_per_type)."""
    nn = tree["num_nodes"]
    out = np.zeros((nn, prm.nsoft))
    suns = np.ascontiguousarray(tree["suns"], np.int32)
    if lib().or_mass_per_type(nn, _ptr(suns), tree["max_part"], _ptr(np.ascontiguousarray(mass_sorted, np.float64)),
                              _ptr(np.ascontiguousarray(st_sorted, np.uint8)), prm.nsoft, _ptr(out)) != 0:
        raise RuntimeError("child node created before its parent")
    return out


def direct(pos, mass, st, prm, targets):
    use_ewald(prm)
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    st = np.ascontiguousarray(st, np.uint8)
    tg = np.ascontiguousarray(targets, np.int64)
    acc = np.zeros((len(tg), 3))
    pot = np.zeros(len(tg))
    lib().or_direct(len(tg), _ptr(tg), len(mass), _ptr(pos), _ptr(mass), _ptr(st), C.byref(prm), _ptr(acc), _ptr(pot))
    return acc, pot


def gravity_direct(pos, mass, st, prm):
    """gravity_direct (gravdirect.c:61-257): the given particles on each other, tabulated short-range
    factor, in order; what gravity() runs below DIRECT_SUMMATION_THRESHOLD active particles."""
    use_ewald(prm)
    pos = np.ascontiguousarray(pos, np.float64)
    n = len(pos)
    acc = np.zeros((n, 3))
    pot = np.zeros(n)
    lib().or_gravity_direct(n, _ptr(pos), _ptr(np.ascontiguousarray(mass, np.float64)),
                            _ptr(np.ascontiguousarray(st, np.uint8)), C.byref(prm), _ptr(acc), _ptr(pot))
    return acc, pot


class OrTsParams(C.Structure):
    _fields_ = [("eta", C.c_double), ("cf_atime", C.c_double), ("cf_a2inv", C.c_double), ("cf_hubble_a", C.c_double),
                ("dtmax", C.c_double), ("dtmin", C.c_double), ("dtdisp", C.c_double), ("timebase_interval", C.c_double),
                ("timebase", C.c_int64), ("ti_current", C.c_int64), ("nostop", C.c_int), ("pad", C.c_int),
                ("sync", C.c_uint8 * 64)]


def timestep_gravity(acc, mass, st, prm, eta, dtmax, dtmin=0.0, dtdisp=0.0, timebase=1 << 29, ti_current=0,
                     bin_old=None, sync=None, pm=None, ids=None, nostop=False):
    """get_timestep_gravity + the new time bin per particle (timestep.c:284-353, 725-770), TimeMax - TimeBegin = 1.
    Returns (ti_step, bin, status) with status 0 or the reference's stop code."""
    acc = np.ascontiguousarray(acc, np.float64)
    n = len(acc)
    t = OrTsParams(eta=eta, cf_atime=1.0, cf_a2inv=1.0, cf_hubble_a=1.0, dtmax=dtmax, dtmin=dtmin, dtdisp=dtdisp,
                   timebase_interval=1.0 / timebase, timebase=timebase, ti_current=ti_current, nostop=int(nostop))
    for b in range(64):
        t.sync[b] = 1 if (sync is None or sync[b]) else 0
    bo = np.zeros(n, np.int8) if bin_old is None else np.ascontiguousarray(bin_old, np.int8)
    ti = np.zeros(n, np.int64)
    bn = np.zeros(n, np.int8)
    pmv = None if pm is None else np.ascontiguousarray(pm, np.float64)
    idv = None if ids is None else np.ascontiguousarray(ids, np.uint64)
    s = lib().or_timestep_gravity(n, _ptr(acc), _ptr(pmv), _ptr(np.ascontiguousarray(mass, np.float64)), _ptr(idv),
                                  _ptr(np.ascontiguousarray(st, np.uint8)), C.byref(prm), C.byref(t), _ptr(bo), _ptr(ti),
                                  _ptr(bn))
    return ti, bn, s


def shortrange_table(rcut_cells: float = 4.5):
    f = np.zeros(NTAB + 1, np.float32)
    p = np.zeros(NTAB + 1, np.float32)
    lib().or_shortrange_table(rcut_cells, _ptr(f), _ptr(p))
    return f, p


def dfs_sequence(tree):
    """Entries in traversal order following nextnode/Nextnode from the root: list of
    ints (>= max_part: node index; < max_part: sorted particle index)."""
    seq = []
    no = tree["max_part"]
    mp = tree["max_part"]
    while no >= 0:
        seq.append(no)
        no = tree["nextnode"][no - mp] if no >= mp else tree["p_next"][no]
    return np.array(seq, np.int64)


def pipeline(pos, mass, st, prm, top=None, passes=2, walk_targets=None):
    """Full single-rank force computation (what gravity() runs on the first step):
    extent, keys, stable sort, top tree, build, BH pass, OldAcc, rebuild, relative pass.
    Returns a dict of every intermediate, in sorted order unless noted."""
    pos = wrap(pos, prm)
    dom = extent(pos, prm)
    hi, lo, ip = keys(pos, prm, dom)
    perm = sort(hi, lo)
    hi_s, lo_s, ip_s = hi[perm], lo[perm], ip[perm]
    pos_s, mass_s, st_s = pos[perm], np.asarray(mass, np.float64)[perm], np.asarray(st, np.uint8)[perm]
    if top is None:
        top = toptree(hi_s, lo_s, prm)
    tree = build(pos_s, mass_s, st_s, ip_s, prm, dom, top)
    out = dict(domain=dom, key_hi=hi, key_lo=lo, perm=perm, top=top, tree=tree, pos_sorted=pos_s, mass_sorted=mass_s,
               st_sorted=st_s, intpos_sorted=ip_s)
    oldacc = np.zeros(len(mass_s), np.float32)
    theta = prm.theta
    for ps in range(passes):
        acc, pot, ni = walk(tree, pos_s, mass_s, st_s, oldacc, prm, walk_targets)
        out[f"acc{ps}"], out[f"pot{ps}"], out[f"ninter{ps}"] = acc, pot, ni
        if walk_targets is None:
            # gravity_force_finalize (src/gravity/accel.c:237-255) with no PM contribution
            oldacc = np.sqrt(acc[:, 0] * acc[:, 0] + acc[:, 1] * acc[:, 1] + acc[:, 2] * acc[:, 2]).astype(np.float32)
            out[f"oldacc{ps}"] = oldacc
        prm.theta = 0.0  # gravity_tree switches to the relative criterion (src/gravity/gravtree.c:654-655)
    prm.theta = theta
    return out


# --------------------------------------------------------------------------------------
# reference harness I/O
# --------------------------------------------------------------------------------------

def write_input(path, pos, mass, st):
    with open(path, "wb") as f:
        np.array([len(mass)], np.int64).tofile(f)
        np.ascontiguousarray(pos, np.float64).tofile(f)
        np.ascontiguousarray(mass, np.float64).tofile(f)
        np.ascontiguousarray(st, np.uint8).tofile(f)


def read_output(path):
    data = open(path, "rb").read()
    assert data[:8] == b"GGREFOUT", "not a harness output"
    off, out = 8, {}
    while off < len(data):
        name = data[off:off + 16].rstrip(b"\0").decode()
        nb = int(np.frombuffer(data, np.int64, 1, off + 16)[0])
        off += 24
        if name == "end":
            break
        out[name] = data[off:off + nb]
        off += nb
    r = {}
    r["domain"] = np.frombuffer(out["domain"], np.float64)
    r["order"] = np.frombuffer(out["order"], np.int64)
    k = np.frombuffer(out["keys"], np.uint64).reshape(-1, 2)
    r["key_hi"], r["key_lo"] = k[:, 0].copy(), k[:, 1].copy()
    r["top"] = np.frombuffer(out["topnodes"], TOPNODE_DTYPE).copy()
    if "order_end" in out:
        r["order_end"] = np.frombuffer(out["order_end"], np.int64)
    if "gravpm" in out:
        r["gravpm"] = np.frombuffer(out["gravpm"], np.float64).reshape(-1, 3)
        r["pmpot"] = np.frombuffer(out["pmpot"], np.float64) if "pmpot" in out else None
    if "tistep" in out:
        r["tistep"] = np.frombuffer(out["tistep"], np.int64)
        r["tbin"] = np.frombuffer(out["tbin"], np.int32)
    if "tree_meta" in out:
        meta = np.frombuffer(out["tree_meta"], np.int64)
        r["tree_meta"] = dict(max_part=int(meta[0]), max_nodes=int(meta[1]), num_nodes=int(meta[2]),
                              first_non_top=int(meta[3]), ntopnodes=int(meta[4]), ntopleaves=int(meta[5]))
        f = np.frombuffer(out["node_f64"], np.float64).reshape(-1, 8)
        i = np.frombuffer(out["node_i32"], np.int32).reshape(-1, 4)
        r["node_center"], r["node_len"], r["node_s"], r["node_mass"] = f[:, 0:3], f[:, 3], f[:, 4:7], f[:, 7]
        r["node_sibling"], r["node_nextnode"], r["node_father"], r["node_maxsoft"] = i[:, 0], i[:, 1], i[:, 2], i[:, 3]
        if "node_mpt" in out:
            r["node_mpt"] = np.frombuffer(out["node_mpt"], np.float64).reshape(len(f), -1)
        r["p_next"] = np.frombuffer(out["nextnode"], np.int32)
        r["p_father"] = np.frombuffer(out["father"], np.int32)
    for ps in range(4):
        if f"acc{ps}" not in out:
            break
        r[f"acc{ps}"] = np.frombuffer(out[f"acc{ps}"], np.float64).reshape(-1, 3)
        r[f"pot{ps}"] = np.frombuffer(out[f"pot{ps}"], np.float64)
        r[f"ninter{ps}"] = np.frombuffer(out[f"ninter{ps}"], np.int32)
        if f"gacc{ps}" in out:
            r[f"gacc{ps}"] = np.frombuffer(out[f"gacc{ps}"], np.float64).reshape(-1, 3)
        r[f"oldacc{ps}"] = np.frombuffer(out[f"oldacc{ps}"], np.float32)
        r[f"time{ps}"] = np.frombuffer(out[f"time{ps}"], np.float64)
    return r


def run_ref(pos, mass, st, periodic, *, box=1.0, asmth=None, rcut=None, theta=0.7, erracc=0.0025,
            softening=(0.01, 0.01), mdom=8, tnf=2.5, passes=2, dump=1, gt=1, first=0, count=None, stride=1,
            timeout=3600, ewald=False, ewald_table_out=None, mns=False, gpu=0, active=1, displace=0.0, minangle=False,
            direct=0, tstep=None, pm=False):
    """Run the compiled reference harness; returns the parsed dump.  tstep: dict(eta=, dtmax=, dtmin=,
    dtdisp=) runs the time-step criterion on the final accelerations (TimeMax = 1, Ti_Current = 0).  ewald=True: the periodic
    pure-tree build (no PM, Ewald correction); its table file is cached in oracle/_ref/ewald_cache
    (the reference writes it to the working directory), ewald_table_out dumps the scaled table.
    gpu=1|2: the harness build whose gravity() step goes through the library's C binding
    (oracle/ref/gpu_gravity.c) with the FP64 or FP32 walk; active=k: every k-th particle in the active
    time bin; displace=f: particle 0 moved outside the domain box before the first pass."""
    if minangle and not (periodic and not ewald and not mns):
        raise ValueError("the ACTIVATE_MINIMUM_OPENING_ANGLE harness is a periodic TreePM build")
    if mns and not (periodic and not ewald):
        raise ValueError("the MULTIPLE_NODE_SOFTENING harness is a periodic TreePM build")
    exe = os.path.join(REF_DIR, "ref_harness_ewald" if ewald else
                       ("ref_harness_pm_mns" if mns else ("ref_harness_pm_mina" if minangle else
                                                          "ref_harness_pmfft" if pm else
                                                           ("ref_harness_pm" if periodic else "ref_harness_iso"))))
    if gpu:
        exe += "_gpu"

    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    cwd = None
    if ewald:
        cwd = os.path.join(REF_DIR, "ewald_cache")
        os.makedirs(cwd, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(fin, pos, mass, st)
        eps = list(softening) + [softening[-1]] * (2 - len(softening))
        args = [exe, fin, fout, f"box={box!r}", f"theta={theta!r}", f"erracc={erracc!r}", f"eps0={eps[0]!r}",
                f"eps1={eps[1]!r}", f"mdom={mdom}", f"tnf={tnf!r}", f"passes={passes}", f"dump={dump}", f"gt={gt}",
                f"first={first}", f"stride={stride}", f"gpu={gpu}", f"active={active}", f"displace={displace!r}", f"direct={direct}"]
        if tstep:
            args += ["tstep=1"] + [f"{k}={v!r}" for k, v in tstep.items()]
        if pm:
            args += ["pm=1"]
        if count is not None:
            args.append(f"count={count}")
        if periodic and not ewald:
            args += [f"asmth={asmth!r}", f"rcut={rcut!r}"]
        if ewald_table_out:
            args.append(f"ewaldout={ewald_table_out}")
        res = subprocess.run(args, capture_output=True, text=True, timeout=timeout, cwd=cwd)
        if res.returncode != 0:
            raise RuntimeError(f"reference harness failed ({res.returncode}): {res.stdout[-2000:]} {res.stderr[-2000:]}")
        out = read_output(fout)
        out["stdout"] = res.stdout
        return out
