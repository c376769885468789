"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the reference's periodic PM long-range force
(src/gravity/pm/pm_periodic.c, pmforce_periodic with the uniform (non-zoom) data path), and the
analytic long-range force it approximates.

Only ``tests/`` import this module; the library under ``arepo_b200/`` never does.

Parity status: pinned to the reference.  FFTW is not in this image, but the reference's own
pm_periodic.c compiles into a harness build (oracle/ref, config_pmfft.h) whose few FFTW calls are
served by oracle/ref/fftw_shim.c (a radix-2 FFT); ``pm_periodic`` agrees with that build's
pmforce_periodic to ~1e-15 of the RMS force (tests/test_pm_oracle.py).  It is also checked against
physics: ``longrange_ewald`` is the reciprocal-space Ewald sum with the same Gaussian split
(alpha = 1 / (2 Asmth), the long-range half of the erfc kernel of the tree walk,
src/gravity/forcetree_walk.c:72-85), evaluated exactly by summing over wave vectors.
"""
from __future__ import annotations

import numpy as np


def _cic(pos, box, n):
    """Cell index and offset per axis: slab = (int)(to_slab_fac * pos), d = to_slab_fac * pos - slab,
    wrapped at the grid size (pm_periodic.c:1090-1120, 1334-1357)."""
    f = n / box
    s = np.floor(f * pos).astype(np.int64)  # positions are >= 0: (int) truncation == floor
    d = f * pos - s
    s0 = s % n
    s1 = (s0 + 1) % n
    return s0, s1, d


def pm_periodic(pos, mass, box, pmgrid, asmth, want_pot=True):
    """Accelerations (and potentials) of the long-range PM force with G = 1, as pmforce_periodic
    (pm_periodic.c:1572-1936): CIC mass assignment, forward FFT, Green's function
    -exp(-k^2 Asmth^2) / k^2 with the CIC deconvolution sinc^-4 (:1644-1699), inverse FFT,
    4-point finite differences of the potential (:1735-1790), CIC readout (:1322-1538)."""
    pos = np.asarray(pos, np.float64)
    mass = np.asarray(mass, np.float64)
    n = pmgrid
    d = box / n
    s0, s1, w = _cic(pos, box, n)
    rho = np.zeros((n, n, n))
    for cx, wx in ((s0[:, 0], 1 - w[:, 0]), (s1[:, 0], w[:, 0])):
        for cy, wy in ((s0[:, 1], 1 - w[:, 1]), (s1[:, 1], w[:, 1])):
            for cz, wz in ((s0[:, 2], 1 - w[:, 2]), (s1[:, 2], w[:, 2])):
                np.add.at(rho, (cx, cy, cz), mass * wx * wy * wz)
    rhok = np.fft.rfftn(rho)  # FFTW forward (unnormalised, e^{-ikx})
    kfac = 2.0 * np.pi / (n * d)
    idx = np.arange(n)
    ii = np.where(idx >= n // 2, idx - n, idx)
    kx = kfac * ii[:, None, None]
    ky = kfac * ii[None, :, None]
    kz = kfac * np.arange(n // 2 + 1)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz

    def sinc(k):
        a = k * 0.5 * d
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(a != 0, np.sin(a) / np.where(a != 0, a, 1.0), 1.0)

    with np.errstate(divide="ignore", invalid="ignore"):
        smth = np.where(k2 > 0, -np.exp(-k2 * asmth * asmth) / np.where(k2 > 0, k2, 1.0), 0.0)
    ff = 1.0 / (sinc(kx) * sinc(ky) * sinc(kz))
    rhok = rhok * (smth * ff ** 4)
    rhok[0, 0, 0] = 0.0
    phi = np.fft.irfftn(rhok, s=(n, n, n), axes=(0, 1, 2)) * (n ** 3)  # FFTW backward is unnormalised
    fac_pot = 4.0 * np.pi / box ** 3
    fac = fac_pot / (2.0 * d)
    acc = np.zeros((len(mass), 3))
    for dim in range(3):
        fg = fac * ((4.0 / 3.0) * (np.roll(phi, 1, axis=dim) - np.roll(phi, -1, axis=dim)) -
                    (1.0 / 6.0) * (np.roll(phi, 2, axis=dim) - np.roll(phi, -2, axis=dim)))
        acc[:, dim] = _readout(fg, s0, s1, w)
    pot = _readout(phi, s0, s1, w) * fac_pot if want_pot else None
    return acc, pot


def _readout(grid, s0, s1, w):
    v = np.zeros(len(w))
    for cx, wx in ((s0[:, 0], 1 - w[:, 0]), (s1[:, 0], w[:, 0])):
        for cy, wy in ((s0[:, 1], 1 - w[:, 1]), (s1[:, 1], w[:, 1])):
            for cz, wz in ((s0[:, 2], 1 - w[:, 2]), (s1[:, 2], w[:, 2])):
                v += grid[cx, cy, cz] * wx * wy * wz
    return v


def longrange_ewald(pos, mass, box, asmth, targets=None, kmax_sigma=6.0):
    """Exact long-range (reciprocal-space) acceleration and potential with G = 1 at `targets`
    (indices) from all particles and their periodic images:
    a_i = -(4 pi / L^3) sum_{k != 0} k exp(-k^2 Asmth^2) / k^2 sum_j m_j sin(k . (x_i - x_j)),
    phi_i = -(4 pi / L^3) sum_{k != 0} exp(-k^2 Asmth^2) / k^2 sum_j m_j cos(k . (x_i - x_j)),
    wave vectors up to |k| Asmth = kmax_sigma."""
    pos = np.asarray(pos, np.float64)
    mass = np.asarray(mass, np.float64)
    t = np.arange(len(mass)) if targets is None else np.asarray(targets)
    kf = 2.0 * np.pi / box
    nmax = int(np.ceil(kmax_sigma / (asmth * kf)))
    r = np.arange(-nmax, nmax + 1)
    K = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3).astype(np.float64) * kf
    k2 = np.sum(K * K, axis=1)
    keep = (k2 > 0) & (k2 * asmth * asmth <= kmax_sigma ** 2)
    K, k2 = K[keep], k2[keep]
    g = np.exp(-k2 * asmth * asmth) / k2
    # structure factor S(k) = sum_j m_j e^{-i k.x_j}; sum_j m_j sin(k.(x_i - x_j)) = Im(e^{i k.x_i} S(k))
    acc = np.zeros((len(t), 3))
    pot = np.zeros(len(t))
    for c0 in range(0, len(K), 4096):
        Kc, gc = K[c0:c0 + 4096], g[c0:c0 + 4096]
        S = np.exp(-1j * (pos @ Kc.T)).T @ mass
        z = np.exp(1j * (pos[t] @ Kc.T)) * S[None, :]
        acc -= (np.imag(z) * gc[None, :]) @ Kc
        pot -= np.real(z) @ gc
    f = 4.0 * np.pi / box ** 3
    return acc * f, pot * f
