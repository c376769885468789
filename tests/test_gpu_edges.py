"""Edge cases of the tree path on the GPU: inputs smaller than one walk group (down to the two
particles the library accepts), particles of zero mass among the sources (the reference skips them
as interaction partners, `forcetree_walk.c:363`, but still computes their own force), and the
sizes the entry points refuse.

The FP64 walk is compared with the oracle bit for bit; the FP32 group walk against the FP64
direct sum, with the tolerance of the other FP32 tests."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200.gravity import GravityTree
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = (2, 3, 7, 31, 33, 97)


def _case(n, periodic):
    rng = np.random.default_rng(n + (1000 if periodic else 0))
    pos = rng.uniform(0.2, 0.8, (n, 3))
    mass = rng.uniform(0.5, 1.5, n) / n
    if n > 3:
        mass[::5] = 0.0
    st = (rng.uniform(size=n) < 0.5).astype(np.uint8)
    a = 1.25 / 16
    p = dict(periodic=periodic, box=1.0, asmth=a if periodic else 0.0, rcut=4.5 * a if periodic else 0.0, rcut_cells=4.5,
             softening=(0.01, 0.02), theta=0.7, erracc=0.0025, mdom=8, tnf=2.5)
    return pos, mass, st, p


def _gpu_params(p, precision):
    return L.make_params(periodic=p["periodic"], box_size=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                         rcut_cells=p["rcut_cells"], softening=p["softening"], err_tol_theta=p["theta"],
                         err_tol_force_acc=p["erracc"], top_node_factor=p["tnf"], multiple_domains=p["mdom"],
                         precision=precision)


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", SIZES)
def test_tiny_inputs_bitexact_vs_oracle(n, periodic, cuda_lib):
    pos, mass, st, p = _case(n, periodic)
    ref = O.pipeline(pos, mass, st, O.make_params(p["periodic"], box=p["box"], asmth=p["asmth"], rcut=p["rcut"],
                                                  rcut_cells=p["rcut_cells"], theta=p["theta"], erracc=p["erracc"],
                                                  softening=p["softening"], mdom=p["mdom"], tnf=p["tnf"]))
    with GravityTree(_gpu_params(p, L.PREC_FP64)) as t:
        acc, pot, ni, old = t.compute_grav_accelerations(pos, mass, st)
        order = t.order()
    assert np.array_equal(order, ref["perm"])
    assert np.array_equal(old[order], ref["oldacc0"])
    assert np.array_equal(acc[order], ref["acc1"])
    assert np.array_equal(pot[order], ref["pot1"])
    assert np.array_equal(ni[order], ref["ninter1"])


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", SIZES)
def test_tiny_inputs_fp32_walk(n, periodic, cuda_lib):
    pos, mass, st, p = _case(n, periodic)
    tg = np.arange(n)
    out = {}
    for prec in (L.PREC_FP64, L.PREC_FP32):
        with GravityTree(_gpu_params(p, prec)) as t:
            acc, pot, ni, _ = t.compute_grav_accelerations(pos, mass, st)
            d, _ = t.direct(tg, cut=True)
        out[prec] = (acc, ni, d)
    d = out[L.PREC_FP64][2]
    scale = np.sqrt(np.mean(np.sum(d * d, axis=1)))

    def err(a):
        return float(np.sqrt(np.mean(np.sum((a - d) ** 2, axis=1))) / scale)

    a32 = out[L.PREC_FP32][0]
    assert np.all(np.isfinite(a32))
    assert err(a32) <= err(out[L.PREC_FP64][0]) * 1.02 + 2e-5
    assert out[L.PREC_FP32][1].sum() >= out[L.PREC_FP64][1].sum()


@pytest.mark.parametrize("n", [0, 1])
def test_fewer_than_two_particles_rejected(n, cuda_lib):
    pos, mass, st, p = _case(2, True)
    with GravityTree(_gpu_params(p, L.PREC_FP64)) as t:
        with pytest.raises(L.GpuGravError) as e:
            t.compute_grav_accelerations(pos[:n], mass[:n], st[:n])
        assert e.value.status == L.ERR_INVALID
