"""The numpy restatement of the reference's periodic PM force (oracle/pm_oracle.py) pinned to
physics: its accelerations and potentials against the exact reciprocal-space Ewald sum with the
same Gaussian split, with the errors shrinking as the split scale grows relative to the mesh
(CIC aliasing and finite-difference truncation), and momentum conserved."""
import os

import numpy as np
import pytest

from oracle import pm_oracle as P


def _rel(a, ref):
    scale = np.sqrt(np.mean(np.sum(ref * ref, axis=-1) if ref.ndim == 2 else ref * ref))
    d = np.linalg.norm(a - ref, axis=1) if a.ndim == 2 else np.abs(a - ref)
    return float(np.sqrt(np.mean(d * d)) / scale)


@pytest.mark.parametrize("cells,tol", [(1.25, 0.025), (3.0, 0.005)])
def test_pm_oracle_matches_ewald_longrange(cells, tol):
    rng = np.random.default_rng(11)
    n, grid = 300, 32
    pos = rng.uniform(0, 1, (n, 3))
    mass = rng.uniform(0.5, 1.5, n) / n
    asmth = cells / grid
    a, p = P.pm_periodic(pos, mass, 1.0, grid, asmth)
    e, ep = P.longrange_ewald(pos, mass, 1.0, asmth)
    assert _rel(a, e) < tol
    assert _rel(p, ep) < tol
    # pairwise forces of a mesh method are antisymmetric: total momentum change vanishes
    tot = np.abs((mass[:, None] * a).sum(0)).max()
    assert tot < 1e-12 * np.abs(mass[:, None] * a).sum()


def test_pm_oracle_box_scaling():
    """Lengths in a box of size L: accelerations scale as 1/L^2 (G M / r^2)."""
    rng = np.random.default_rng(12)
    pos = rng.uniform(0, 1, (200, 3))
    mass = np.full(200, 1.0 / 200)
    a1, _ = P.pm_periodic(pos, mass, 1.0, 32, 1.25 / 32)
    a3, _ = P.pm_periodic(3.0 * pos, mass, 3.0, 32, 3.0 * 1.25 / 32)
    assert np.allclose(a3 * 9.0, a1, rtol=1e-9, atol=1e-12 * np.abs(a1).max())


def test_pm_oracle_matches_reference_pmforce_periodic():
    """The restatement against the reference's own pmforce_periodic (gravity/pm/pm_periodic.c, built
    into the harness with its FFTW calls served by oracle/ref/fftw_shim.c) on the 32^3 grid box at
    PMGRID 64: agreement to the rounding of two FFT implementations (1e-12 of the RMS force)."""
    from oracle import oracle as O

    if not os.path.exists(os.path.join(O.REF_DIR, "ref_harness_pmfft")):
        pytest.skip("reference harness with the periodic PM not built")
    from arepo_b200 import ics

    ic = ics.grid_box(n1=32, sigma_cells=0.2, seed=1001, pmgrid=64)
    soft = (ic["softening"][0],) * 2
    r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft, dump=0,
                  gt=0, pm=True, passes=1)
    o = r["order_end"]
    pos = O.wrap(ic["pos"], O.make_params(True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft))
    a, p = P.pm_periodic(pos[o], ic["mass"][o], 1.0, 64, ic["asmth"])
    assert _rel(a, r["gravpm"]) < 1e-12
    assert _rel(p, r["pmpot"]) < 1e-12
