"""Seeded synthetic particle sets for the workloads of this engine.

There is no network and no initial-condition file of the right size in the
image, so every workload is generated here from a fixed numpy PCG64 seed with
the shapes, sizes and value distributions the workload names:

  grid_box        N = n1^3 regular grid + Gaussian displacements (periodic, L=1)
  hernquist       isolated Hernquist halo, a=1, M=1, truncated at 50a
  zeldovich_box   N = n1^3 grid + Zel'dovich displacements of a P(k) ~ k^-2 field
  zoom_box        2^k uniform low-res particles (mass 8m) + 2^k Plummer high-res (mass m)
  plummer         Plummer sphere, b=1, M=1 (serving stream)

Each returns a dict with pos (n,3) float64, mass (n,) float64, softtype (n,)
uint8 and the run parameters that go with it (periodic, box, asmth, rcut,
softening per type).
"""
from __future__ import annotations

import numpy as np

ASMTH = 1.25  # ASMTH default (src/main/allvars.h:457-462)
RCUT = 4.5    # RCUT default (src/main/allvars.h:464-470)


def _treepm(pmgrid: int, box: float = 1.0):
    asmth = ASMTH * box / pmgrid  # All.Asmth[0], src/gravity/pm/pm_periodic.c:190
    return dict(periodic=True, box=box, asmth=asmth, rcut=RCUT * asmth)  # All.Rcut[0], :191


def grid_box(n1: int = 32, sigma_cells: float = 0.2, seed: int = 1001, pmgrid: int = 64, soft_frac: float = 1 / 40):
    rng = np.random.default_rng(seed)
    g = (np.indices((n1, n1, n1)).reshape(3, -1).T + 0.5) / n1
    pos = np.mod(g + rng.normal(0.0, sigma_cells / n1, g.shape), 1.0)
    n = n1 ** 3
    d = dict(pos=pos, mass=np.full(n, 1.0 / n), softtype=np.zeros(n, np.uint8), softening=(soft_frac / n1,))
    d.update(_treepm(pmgrid))
    return d


def hernquist(n: int = 1 << 20, seed: int = 1002, a: float = 1.0, rmax_a: float = 50.0, eps: float = 0.01):
    rng = np.random.default_rng(seed)
    rmax = rmax_a * a
    mmax = rmax ** 2 / (rmax + a) ** 2  # M(r) = r^2/(r+a)^2 for M=1
    u = rng.uniform(0.0, mmax, n)
    su = np.sqrt(u)
    r = a * su / (1.0 - su)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    pos = r[:, None] * v
    return dict(pos=pos, mass=np.full(n, 1.0 / n), softtype=np.zeros(n, np.uint8), softening=(eps * a,), periodic=False,
                box=1.0, asmth=0.0, rcut=0.0)


def plummer_positions(rng, n: int, b: float, rtrunc: float | None = None) -> np.ndarray:
    out = np.empty((0, 3))
    while len(out) < n:
        m = n - len(out)
        u = rng.uniform(1e-12, 1.0, int(m * 1.3) + 16)
        r = b / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        if rtrunc is not None:
            r = r[r < rtrunc]
        v = rng.normal(size=(len(r), 3))
        v /= np.linalg.norm(v, axis=1)[:, None]
        out = np.concatenate([out, r[:, None] * v])
    return out[:n]


def plummer(n: int, seed: int, b: float = 1.0, eps: float = 0.02):
    rng = np.random.default_rng(seed)
    pos = plummer_positions(rng, n, b)
    return dict(pos=pos, mass=np.full(n, 1.0 / n), softtype=np.zeros(n, np.uint8), softening=(eps * b,), periodic=False,
                box=1.0, asmth=0.0, rcut=0.0)


def zeldovich_box(n1: int = 256, seed: int = 1003, pmgrid: int = 512, rms_cells: float = 0.5, soft_frac: float = 1 / 30):
    """Grid + Zel'dovich displacement psi(k) = i k / k^2 delta(k), P(k) ~ k^-2 up to the
    grid Nyquist frequency, normalised to an rms displacement of rms_cells grid spacings."""
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n1) * n1
    kz1 = np.fft.rfftfreq(n1) * n1
    kx, ky, kz = np.meshgrid(k1, k1, kz1, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = np.sqrt(k2 ** -1.0)  # sqrt(P(k)), P ~ k^-2
    amp[0, 0, 0] = 0.0
    nyq = n1 // 2
    amp[(np.abs(kx) >= nyq) | (np.abs(ky) >= nyq) | (np.abs(kz) >= nyq)] = 0.0
    delta_k = (rng.normal(size=amp.shape) + 1j * rng.normal(size=amp.shape)) * amp
    pos = (np.indices((n1, n1, n1)).reshape(3, -1).T.astype(np.float64) + 0.5) / n1
    disp = np.empty_like(pos)
    for ax, kk in enumerate((kx, ky, kz)):
        psi_k = 1j * kk / k2 * delta_k
        disp[:, ax] = np.fft.irfftn(psi_k, s=(n1, n1, n1)).reshape(-1)
    disp *= (rms_cells / n1) / np.sqrt(np.mean(np.sum(disp * disp, axis=1)))
    pos = np.mod(pos + disp, 1.0)
    n = n1 ** 3
    d = dict(pos=pos, mass=np.full(n, 1.0 / n), softtype=np.zeros(n, np.uint8), softening=(soft_frac / n1,))
    d.update(_treepm(pmgrid))
    return d


def zoom_box_softening(log2_half: int = 23, b: float = 0.02):
    """Plummer-equivalent softening of the zoom box's two species: 1/40 of the mean spacing of the
    uniform particles, and of the Plummer particles inside the half-mass radius 1.305 b."""
    nh = 1 << log2_half
    v_half = 4.0 / 3.0 * np.pi * (1.305 * b) ** 3
    return ((1.0 / nh) ** (1.0 / 3.0) / 40.0, (v_half / (nh / 2)) ** (1.0 / 3.0) / 40.0)


def zoom_box(log2_half: int = 23, seed: int = 1004, pmgrid: int = 512, b: float = 0.02, rtrunc: float = 0.1):
    """2^k low-resolution particles of mass 8m uniform in L=1 and 2^k high-resolution
    particles of mass m, Plummer (scale b) truncated at rtrunc around the box centre.
    Softening 1/40 of the local mean spacing per species (softening types 0 and 1)."""
    nh = 1 << log2_half
    rng_lo = np.random.default_rng([seed, 0])
    rng_hi = np.random.default_rng([seed, 1])
    lo = rng_lo.uniform(0.0, 1.0, (nh, 3))
    hi = np.mod(0.5 + plummer_positions(rng_hi, nh, b, rtrunc), 1.0)
    m = 1.0 / (9.0 * nh)
    pos = np.concatenate([lo, hi])
    mass = np.concatenate([np.full(nh, 8.0 * m), np.full(nh, m)])
    st = np.concatenate([np.zeros(nh, np.uint8), np.ones(nh, np.uint8)])
    d = dict(pos=pos, mass=mass, softtype=st, softening=zoom_box_softening(log2_half, b))
    d.update(_treepm(pmgrid))
    return d


def params_for(ic: dict, **kw):
    """gpugrav_params for a generated set."""
    from ._lib import make_params

    return make_params(
        periodic=ic["periodic"], box_size=ic["box"], asmth=ic["asmth"], rcut=ic["rcut"], rcut_cells=RCUT,
        softening=ic["softening"], **kw,
    )
