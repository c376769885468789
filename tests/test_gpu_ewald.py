"""Periodic box without PM (asmth = 0): the walks add the reference's Ewald correction per
interaction.  The FP64 walk is compared bit for bit with the oracle (which the CPU tests pin to the
reference, tables included); the FP64 direct sum with the same correction against an exact Ewald
sum; the FP32 walk against the FP64 walk; caller-supplied tables against the built-in ones."""
import numpy as np
import pytest
from scipy.special import erfc

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from oracle import oracle as O
from oracle import pm_oracle as P

pytestmark = pytest.mark.gpu

BOX = 2.0


def _params(precision=L.PREC_FP64, eps=0.004, erracc=0.0025):
    return L.make_params(periodic=True, box_size=BOX, asmth=0.0, rcut=0.0, softening=(eps,), precision=precision,
                         err_tol_force_acc=erracc)


def _clustered(n, seed):
    rng = np.random.default_rng(seed)
    k = n // 2
    pos = np.concatenate([rng.uniform(0, BOX, (n - k, 3)), (1.3 + ics.plummer_positions(rng, k, 0.05, 0.4)) % BOX])
    return pos, np.full(n, 1.0 / n), np.zeros(n, np.uint8)


def test_fp64_ewald_walk_bitexact_vs_oracle(cuda_lib):
    pos, mass, st = _clustered(20000, 31)
    with GravityTree(_params()) as t:
        acc, pot, ni, old = t.compute_grav_accelerations(pos, mass, st)
        order = t.order()
    oprm = O.make_params(True, box=BOX, asmth=0.0, rcut=0.0, softening=(0.004,))
    ref = O.pipeline(pos, mass, st, oprm)
    assert np.array_equal(order, ref["perm"])
    assert np.array_equal(old[order], ref["oldacc0"])
    assert np.array_equal(acc[order], ref["acc1"])
    assert np.array_equal(pot[order], ref["pot1"])
    assert np.array_equal(ni[order], ref["ninter1"])


def test_caller_tables_equal_builtin(cuda_lib):
    pos, mass, st = _clustered(5000, 32)
    t0 = O.ewald_table()
    scaled = [t0[0] / BOX ** 2, t0[1] / BOX ** 2, t0[2] / BOX ** 2, t0[3] / BOX]
    with GravityTree(_params()) as t:
        a1, p1, _, _ = t.compute_grav_accelerations(pos, mass, st)
    with GravityTree(_params()) as t:
        t.set_ewald_table(*scaled)
        a2, p2, _, _ = t.compute_grav_accelerations(pos, mass, st)
        assert t.lib.gpugrav_set_ewald_table(t._ctx, 32, None, None, None, None) == L.ERR_INVALID
    assert np.array_equal(a1, a2) and np.array_equal(p1, p2)


def _ewald_exact(pos, mass, box, alpha_len):
    """Newtonian force of all periodic images (G = 1, no softening): Ewald sum with split length
    alpha_len (real space over the 27 nearest cells, reciprocal space exact)."""
    acc = np.zeros_like(pos)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                d = pos[None, :, :] - pos[:, None, :]
                d -= box * np.round(d / box)
                d += box * np.array([sx, sy, sz])
                r2 = np.sum(d * d, axis=2)
                self_ = r2 == 0
                r2[self_] = 1.0
                r = np.sqrt(r2)
                u = r / (2.0 * alpha_len)
                f = (erfc(u) + 2.0 * u / np.sqrt(np.pi) * np.exp(-u * u)) / (r2 * r)
                f[self_] = 0.0
                acc += np.einsum("ij,ijk->ik", f * mass[None, :], d)
    a_long, _ = P.longrange_ewald(pos, mass, box, alpha_len)
    return acc + a_long


def test_ewald_direct_sum_matches_exact_ewald(cuda_lib):
    rng = np.random.default_rng(33)
    n = 400
    pos = rng.uniform(0, BOX, (n, 3))
    mass = rng.uniform(0.5, 1.5, n) / n
    with GravityTree(_params(eps=1e-6)) as t:
        t.domain_decomposition(pos, mass, np.zeros(n, np.uint8))
        d, _ = t.direct(np.arange(n))
    ref = _ewald_exact(pos, mass, BOX, 0.12 * BOX)
    scale = np.sqrt(np.mean(np.sum(ref * ref, axis=1)))
    err = np.linalg.norm(d - ref, axis=1) / scale
    assert np.max(err) < 2e-4  # trilinear interpolation of the tables (64 cells per half box)


def test_fp32_ewald_walk_accuracy(cuda_lib):
    pos, mass, st = _clustered(30000, 34)
    tg = np.sort(np.random.default_rng(35).choice(len(mass), 2048, replace=False))
    out = {}
    for prec in (L.PREC_FP64, L.PREC_FP32):
        with GravityTree(_params(precision=prec)) as t:
            acc, _, ni, _ = t.compute_grav_accelerations(pos, mass, st)
            d, _ = t.direct(tg)
        out[prec] = (acc, ni, d)
    d = out[L.PREC_FP64][2]
    scale = np.sqrt(np.mean(np.sum(d * d, axis=1)))

    def err(a):
        return float(np.sqrt(np.mean(np.sum((a[tg] - d) ** 2, axis=1))) / scale)

    e64, e32 = err(out[L.PREC_FP64][0]), err(out[L.PREC_FP32][0])
    assert e32 <= e64 * 1.02 + 2e-5, (e32, e64)
    assert e32 < 5e-3
    assert out[L.PREC_FP32][1].sum() >= out[L.PREC_FP64][1].sum()
