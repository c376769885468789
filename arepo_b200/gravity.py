"""Host-side interface of the B200 tree-gravity engine, shaped like the
reference's gravity driver.

    reference (src/gravity/accel.c:58-80, 94-192)        here
    ----------------------------------------------       -------------------------------
    domain_Decomposition()   [keys + sort part]          GravityTree.domain_decomposition()
    construct_forcetree(0, ...)                          GravityTree.construct_forcetree()
    gravity_tree(timebin)                                GravityTree.gravity_tree()
    compute_grav_accelerations() on the first step       GravityTree.compute_grav_accelerations()
      (Barnes-Hut pass, OldAcc, relative pass)

Everything runs in libarepo_gpugrav on the GPU; this module only moves
arguments across the C ABI and raises GpuGravError on a negative status (the
reference's -1/-2/-3 codes keep their meaning).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class GravityTree:
    def __init__(self, params: L.Params, device: int = 0):
        self.lib = L.load()
        self.params = params
        self._ctx = C.c_void_p()
        self._check(self.lib.gpugrav_create(C.byref(self._ctx), device, C.byref(params)), ctx=False)
        self.n = 0

    # ---- lifetime ----
    def close(self):
        if self._ctx:
            self.lib.gpugrav_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, status: int, ctx: bool = True):
        if status != L.OK:
            msg = self.lib.gpugrav_status_string(status).decode()
            if ctx and self._ctx:
                msg += ": " + self.lib.gpugrav_last_error(self._ctx).decode()
            raise L.GpuGravError(status, msg)

    def set_params(self, params: L.Params):
        self._check(self.lib.gpugrav_set_params(self._ctx, C.byref(params)))
        self.params = params

    def pm_periodic(self, pmgrid: int, pos, mass, want_pot: bool = True, mem: int = L.MEM_HOST):
        """Long-range periodic PM accelerations (without G) and potentials, as pmforce_periodic
        (src/gravity/pm/pm_periodic.c:1572-1936); uses this context's box_size and asmth."""
        if mem == L.MEM_HOST:
            pos = np.ascontiguousarray(pos, np.float64)
            mass = np.ascontiguousarray(mass, np.float64)
            acc = np.empty((len(mass), 3), np.float64)
            pot = np.empty(len(mass), np.float64) if want_pot else None
        else:
            import torch

            acc = torch.empty((mass.shape[0], 3), dtype=torch.float64, device=pos.device)
            pot = torch.empty(mass.shape[0], dtype=torch.float64, device=pos.device) if want_pot else None
        self._check(self.lib.gpugrav_pm_periodic(self._ctx, pmgrid, len(mass) if mem == L.MEM_HOST else mass.shape[0],
                                                 L.ptr(pos), L.ptr(mass), L.ptr(acc), L.ptr(pot), mem))
        return acc, pot

    def mass_per_type(self) -> np.ndarray:
        """ExtNodes[].mass_per_type of the last build (MULTIPLE_NODE_SOFTENING), reference node order."""
        out = np.empty((self.tree_info().num_nodes, self.params.nsofttypes))
        self._check(self.lib.gpugrav_export_mass_per_type(self._ctx, L.ptr(out)))
        return out

    def set_ewald_table(self, fx, fy, fz, pot):
        """AREPO's Ewald correction tables (Ewd_fcorrx/y/z, Ewd_potcorr after ewald_init: scaled to
        the box), (65, 65, 65) or flat doubles each, for a periodic context without PM (asmth = 0)."""
        arrs = [np.ascontiguousarray(a, np.float64).ravel() for a in (fx, fy, fz, pot)]
        self._check(self.lib.gpugrav_set_ewald_table(self._ctx, 64, *[L.ptr(a) for a in arrs]))

    def set_target_slice(self, slice_: int, nslices: int):
        """Walk only slice `slice_` of `nslices` key-ordered target slices; other targets' outputs
        are zero (the slices of G ranks sum to the full result)."""
        self._check(self.lib.gpugrav_set_target_slice(self._ctx, slice_, nslices))

    def set_target_slice_cost(self, slice_: int, nslices: int, cost=None, mem: int = L.MEM_HOST):
        """Key-ordered target slices of equal cost (per-particle cost in caller order, e.g. the previous
        step's interaction counts); cost None: equal counts."""
        n = 0 if cost is None else (cost.shape[0] if hasattr(cost, "shape") else len(cost))
        if cost is not None and mem == L.MEM_HOST:
            cost = np.ascontiguousarray(cost, np.float32)
        self._check(self.lib.gpugrav_set_target_slice_cost(self._ctx, slice_, nslices, n, L.ptr(cost), mem))

    # cudaStreamLegacy: the legacy default stream as an explicit handle (cuda_runtime_api.h)
    _CUDA_STREAM_LEGACY = 0x1

    def set_stream(self, stream_handle: int | None):
        """Run the context's work on `stream_handle` (a cudaStream_t as an int, e.g. a torch stream's
        `cuda_stream`); None: the context's own stream.  0 is the legacy default stream (torch's default
        stream), which the C ABI takes as cudaStreamLegacy (NULL there means the context's own stream,
        which does not order against the caller's work)."""
        if stream_handle is None:
            h = None
        else:
            h = C.c_void_p(stream_handle if stream_handle != 0 else self._CUDA_STREAM_LEGACY)
        self._check(self.lib.gpugrav_set_stream(self._ctx, h))

    def synchronize(self):
        self._check(self.lib.gpugrav_synchronize(self._ctx))

    # ---- the path ----
    def domain_decomposition(self, pos, mass, softtype, domain: L.Domain | None = None, mem: int = L.MEM_HOST):
        """Wrap, extent (unless `domain` is given), 126-bit keys and stable key sort.
        Host arrays (numpy) with mem=MEM_HOST; device tensors with mem=MEM_DEVICE."""
        if mem == L.MEM_HOST:
            pos = np.ascontiguousarray(pos, np.float64)
            mass = np.ascontiguousarray(mass, np.float64)
            softtype = np.ascontiguousarray(softtype, np.uint8)
        n = len(mass)
        self._keep = (pos, mass, softtype)
        self._check(
            self.lib.gpugrav_load(
                self._ctx, n, L.ptr(pos), L.ptr(mass), L.ptr(softtype), mem, C.byref(domain) if domain is not None else None
            )
        )
        self.n = n

    def construct_forcetree(self, topnodes: np.ndarray | None = None) -> int:
        """Top-level skeleton, octree, moments, threading. Returns Tree_NumNodes."""
        if topnodes is not None:
            top = np.ascontiguousarray(topnodes, L.TOPNODE_DTYPE)
            self._check(self.lib.gpugrav_build(self._ctx, top.ctypes.data_as(C.c_void_p), len(top)))
        else:
            self._check(self.lib.gpugrav_build(self._ctx, None, 0))
        return self.tree_info().num_nodes

    def gravity_tree(self, oldacc=None, acc=None, pot=None, ninter=None, mem: int = L.MEM_HOST, want_pot: bool = True):
        """Accelerations (without G), potentials and interaction counts for every particle,
        in the caller's order. With mem=MEM_HOST numpy outputs are allocated when not given;
        want_pot=False skips the potential (EVALPOTENTIAL off)."""
        n = self.n
        if mem == L.MEM_HOST:
            if acc is None:
                acc = np.empty((n, 3), np.float64)
            if pot is None and want_pot:
                pot = np.empty(n, np.float64)
            if ninter is None:
                ninter = np.empty(n, np.int32)
            if oldacc is not None:
                oldacc = np.ascontiguousarray(oldacc, np.float32)
        self._check(self.lib.gpugrav_walk(self._ctx, L.ptr(oldacc), L.ptr(acc), L.ptr(pot), L.ptr(ninter), mem))
        return acc, pot, ninter

    def gravity_tree_targets(self, targets, oldacc=None, want_pot: bool = True):
        """gravity_tree(timebin) for an active subset: `targets` are caller indices (TargetList,
        src/gravity/gravtree.c:494-520); outputs (host arrays) in the order of `targets`."""
        tg = np.ascontiguousarray(targets, np.int32)
        nt = len(tg)
        acc = np.empty((nt, 3), np.float64)
        pot = np.empty(nt, np.float64) if want_pot else None
        ninter = np.empty(nt, np.int32)
        if oldacc is not None:
            oldacc = np.ascontiguousarray(oldacc, np.float32)
        self._check(self.lib.gpugrav_walk_targets(self._ctx, nt, L.ptr(tg), L.ptr(oldacc), L.ptr(acc), L.ptr(pot),
                                                  L.ptr(ninter), L.MEM_HOST))
        return acc, pot, ninter

    def gravity_direct(self, pos, mass, softtype, want_pot: bool = True):
        """gravity_direct (src/gravity/gravdirect.c:61-257): the given particles on each other by direct
        summation, what gravity() runs below DIRECT_SUMMATION_THRESHOLD active particles."""
        pos = np.ascontiguousarray(pos, np.float64)
        n = len(pos)
        acc = np.empty((n, 3), np.float64)
        pot = np.empty(n, np.float64) if want_pot else None
        self._check(self.lib.gpugrav_gravity_direct(self._ctx, n, L.ptr(pos), L.ptr(np.ascontiguousarray(mass, np.float64)),
                                                    L.ptr(np.ascontiguousarray(softtype, np.uint8)), L.ptr(acc), L.ptr(pot),
                                                    L.MEM_HOST))
        return acc, pot

    def timestep_gravity(self, tp: L.TimestepParams, grav_accel, mass, softtype, bin_old, grav_pm=None, ids=None):
        """get_timestep_gravity + the new TimeBinGrav (timestep.c:284-353, 725-770) per particle:
        returns (ti_step int64, bin int8)."""
        a = np.ascontiguousarray(grav_accel, np.float64)
        n = len(a)
        ti = np.empty(n, np.int64)
        b = np.empty(n, np.int8)
        failed = C.c_int64(-1)
        pm = None if grav_pm is None else np.ascontiguousarray(grav_pm, np.float64)
        idv = None if ids is None else np.ascontiguousarray(ids, np.uint64)
        self._check(self.lib.gpugrav_timestep_gravity(self._ctx, C.byref(tp), n, L.ptr(a), L.ptr(pm),
                                                      L.ptr(np.ascontiguousarray(mass, np.float64)), L.ptr(idv),
                                                      L.ptr(np.ascontiguousarray(softtype, np.uint8)),
                                                      L.ptr(np.ascontiguousarray(bin_old, np.int8)), L.ptr(ti), L.ptr(b),
                                                      C.byref(failed), L.MEM_HOST))
        return ti, b

    def active_particles(self, bins, synchronized):
        """indices of the particles whose time bin is synchronized (TimeBinsGravity.ActiveParticleList)"""
        b = np.ascontiguousarray(bins, np.int8)
        sync = (C.c_uint8 * 64)(*[1 if s else 0 for s in synchronized])
        out = np.empty(len(b), np.int32)
        cnt = C.c_int64(0)
        self._check(self.lib.gpugrav_active_particles(self._ctx, len(b), L.ptr(b), sync, L.ptr(out), C.byref(cnt), L.MEM_HOST))
        return out[: cnt.value].copy()

    def compute_grav_accelerations(self, pos, mass, softtype, topnodes=None, pm_acc=None):
        """First-step sequence of compute_grav_accelerations (src/gravity/accel.c:58-80):
        Barnes-Hut pass, OldAcc = |a_tree + a_PM/G| (gravity_force_finalize, accel.c:237-255),
        then the relative-criterion pass. Returns (acc, pot, ninter, oldacc) of the second pass."""
        self.domain_decomposition(pos, mass, softtype)
        self.construct_forcetree(topnodes)
        p = self.params
        theta = p.err_tol_theta
        acc, pot, ni = self.gravity_tree()
        a = acc if pm_acc is None else acc + pm_acc
        oldacc = np.sqrt(a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1] + a[:, 2] * a[:, 2]).astype(np.float32)
        if p.type_of_opening_criterion == 1:
            p.err_tol_theta = 0.0  # gravity_tree switches to the relative criterion (gravtree.c:654-655)
            self.set_params(p)
            try:
                acc, pot, ni = self.gravity_tree(oldacc)
            finally:
                p.err_tol_theta = theta
                self.set_params(p)
        return acc, pot, ni, oldacc

    # ---- introspection ----
    def domain(self) -> L.Domain:
        d = L.Domain()
        self._check(self.lib.gpugrav_get_domain(self._ctx, C.byref(d)))
        return d

    def order(self) -> np.ndarray:
        o = np.empty(self.n, np.int64)
        self._check(self.lib.gpugrav_get_order(self._ctx, L.ptr(o)))
        return o

    def keys(self):
        hi = np.empty(self.n, np.uint64)
        lo = np.empty(self.n, np.uint64)
        self._check(self.lib.gpugrav_get_keys(self._ctx, L.ptr(hi), L.ptr(lo)))
        return hi, lo

    def topnodes(self) -> np.ndarray:
        nt = C.c_int32()
        self._check(self.lib.gpugrav_get_topnodes(self._ctx, None, 0, C.byref(nt)))
        out = np.zeros(nt.value, L.TOPNODE_DTYPE)
        self._check(self.lib.gpugrav_get_topnodes(self._ctx, out.ctypes.data_as(C.c_void_p), nt.value, C.byref(nt)))
        return out

    def tree_info(self) -> L.TreeInfo:
        t = L.TreeInfo()
        self._check(self.lib.gpugrav_get_tree_info(self._ctx, C.byref(t)))
        return t

    def export_tree(self) -> dict:
        info = self.tree_info()
        nn, n = info.num_nodes, self.n
        t = dict(
            center=np.empty((nn, 3)), len=np.empty(nn), s=np.empty((nn, 3)), mass=np.empty(nn),
            sibling=np.empty(nn, np.int32), nextnode=np.empty(nn, np.int32), father=np.empty(nn, np.int32),
            maxsoft=np.empty(nn, np.uint8), p_next=np.empty(n, np.int32), p_father=np.empty(n, np.int32),
        )
        self._check(self.lib.gpugrav_export_tree(self._ctx, *[L.ptr(t[k]) for k in (
            "center", "len", "s", "mass", "sibling", "nextnode", "father", "maxsoft", "p_next", "p_father")]))
        t.update(num_nodes=int(nn), max_part=int(info.max_part), first_non_top=int(info.first_non_top),
                 max_depth=int(info.max_depth), coincident_cells=int(info.coincident_cells))
        return t

    def timings(self) -> L.Timings:
        t = L.Timings()
        self._check(self.lib.gpugrav_get_timings(self._ctx, C.byref(t)))
        return t

    def direct_split(self, targets):
        """FORCETEST's split (gravtree_forcetest.c:537-620): (acc_total, pot_total, acc_short, pot_short);
        the short-range part only for TreePM contexts (else None)."""
        tg = np.ascontiguousarray(targets, np.int64)
        nt = len(tg)
        at, pt = np.empty((nt, 3)), np.empty(nt)
        treepm = bool(self.params.periodic) and self.params.asmth > 0
        a_s, p_s = (np.empty((nt, 3)), np.empty(nt)) if treepm else (None, None)
        self._check(self.lib.gpugrav_direct_split(self._ctx, nt, L.ptr(tg), L.ptr(at), L.ptr(pt), L.ptr(a_s), L.ptr(p_s)))
        return at, pt, a_s, p_s

    def direct(self, targets, cut: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """FP64 direct summation for the given caller indices (accuracy instrument). cut=True keeps
        only pairs closer than Rcut (the range the walk evaluates) in a periodic TreePM run."""
        tg = np.ascontiguousarray(targets, np.int64)
        acc = np.empty((len(tg), 3))
        pot = np.empty(len(tg))
        self._check(self.lib.gpugrav_direct(self._ctx, len(tg), L.ptr(tg), L.DIRECT_CUT if cut else L.DIRECT_FULL,
                                                    L.ptr(acc), L.ptr(pot)))
        return acc, pot
