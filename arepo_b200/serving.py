"""Serving loop: many independent isolated N-body systems, continuously batched
on one GPU (libarepo_gpugrav's gpugrav_serve_* entry points).

    srv = GravityServer(params, max_systems=4096, max_particles=1 << 26, budget_bytes=120e9)
    srv.submit(request_id, pos, vel, mass, softtype, nsteps=16, dt=0.005)
    while srv.busy():
        srv.tick()                       # one force evaluation for every admitted system
        for res in srv.poll_all():       # finished requests: final pos, vel, acc, timings
            ...

A request runs the reference's first-step sequence (Barnes-Hut pass, OldAcc,
relative pass) and then `nsteps` kick-drift-kick steps.  max_systems=1 runs one
request at a time (the serial baseline).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class ServeResult:
    id: int
    pos: np.ndarray
    vel: np.ndarray
    acc: np.ndarray
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class GravityServer:
    def __init__(self, params: L.Params, device: int = 0, max_systems: int = 4096, max_particles: int = 1 << 24,
                 budget_bytes: float = 0):
        self.lib = L.load()
        cfg = L.ServeConfig()
        cfg.abi_version = L.ABI_VERSION
        cfg.max_systems = max_systems
        cfg.max_particles = int(max_particles)
        cfg.memory_budget_bytes = int(budget_bytes)
        self._srv = C.c_void_p()
        s = self.lib.gpugrav_serve_create(C.byref(self._srv), device, C.byref(params), C.byref(cfg))
        if s != L.OK:
            raise L.GpuGravError(s, self.lib.gpugrav_status_string(s).decode())

    def close(self):
        if self._srv:
            self.lib.gpugrav_serve_destroy(self._srv)
            self._srv = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, s):
        if s != L.OK:
            raise L.GpuGravError(s, self.lib.gpugrav_status_string(s).decode() + ": " +
                                 self.lib.gpugrav_serve_last_error(self._srv).decode())

    def submit(self, rid: int, pos, vel, mass, softtype, nsteps: int, dt: float):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        softtype = np.ascontiguousarray(softtype, np.uint8)
        self._check(self.lib.gpugrav_serve_submit(self._srv, rid, len(mass), L.ptr(pos), L.ptr(vel), L.ptr(mass),
                                                  L.ptr(softtype), nsteps, dt))

    def cancel(self, rid: int):
        self._check(self.lib.gpugrav_serve_cancel(self._srv, rid))

    def tick(self) -> int:
        na = C.c_int32(0)
        self._check(self.lib.gpugrav_serve_tick(self._srv, C.byref(na)))
        return na.value

    def stats(self) -> L.ServeStats:
        st = L.ServeStats()
        self._check(self.lib.gpugrav_serve_get_stats(self._srv, C.byref(st)))
        return st

    def busy(self) -> bool:
        st = self.stats()
        return st.waiting > 0 or st.running > 0

    def poll(self, out=None) -> ServeResult | None:
        """Oldest finished request, or None.  `out` (optional): a mapping from request id to
        caller-owned (pos, vel, acc) float64 arrays of shape (n, 3) that receive the result (no
        allocation per result); ids not in it get new arrays."""
        rid, n = C.c_int64(), C.c_int64()
        self._check(self.lib.gpugrav_serve_poll(self._srv, C.byref(rid), C.byref(n), None, None, None, 0, None))
        if rid.value < 0:
            return None
        bufs = out.get(int(rid.value)) if out is not None else None
        if bufs is not None:
            pos, vel, acc = bufs
            for a in bufs:
                if a.shape != (n.value, 3) or a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError("result buffers must be C-contiguous float64 of shape (n, 3)")
        else:
            pos = np.empty((n.value, 3))
            vel = np.empty((n.value, 3))
            acc = np.empty((n.value, 3))
        times = np.empty(3)
        self._check(self.lib.gpugrav_serve_poll(self._srv, C.byref(rid), C.byref(n), L.ptr(pos), L.ptr(vel), L.ptr(acc),
                                                n.value, L.ptr(times)))
        return ServeResult(int(rid.value), pos, vel, acc, float(times[0]), float(times[1]), float(times[2]))

    def poll_all(self, out=None) -> list[ServeResult]:
        res = []
        while True:
            r = self.poll(out)
            if r is None:
                return res
            res.append(r)

    def run_to_completion(self) -> dict[int, ServeResult]:
        res = {}
        while self.busy():
            self.tick()
            for r in self.poll_all():
                res[r.id] = r
        for r in self.poll_all():
            res[r.id] = r
        return res


def serving_params(softening: float, err_tol_force_acc: float = 0.0025, err_tol_theta: float = 0.7) -> L.Params:
    """Isolated systems, G = 1, one softening type (Plummer-equivalent epsilon)."""
    return L.make_params(periodic=False, softening=(softening,), err_tol_theta=err_tol_theta,
                         err_tol_force_acc=err_tol_force_acc, precision=L.PREC_FP32)
