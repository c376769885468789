"""The drop-in from C: the reference's own gravity step, built twice from its unmodified sources --
once as it is (construct_forcetree + gravity_tree) and once with those two calls replaced by the
library through oracle/ref/gpu_gravity.c, the binding AREPO would compile in under GPU_GRAVITY.
Both run on AREPO's own data structures (P[], All, the domain globals, TopNodes, TimeBinsGravity).

FP64 walk: GravAccel bit-identical in both passes (Barnes-Hut, then relative with the reference's
OldAcc), for every particle, for an active subset of the particles (gravity_tree's TargetList), and
after a particle left the domain box (the binding redoes the domain decomposition on -3 as
force_treebuild does).  FP32 walk: the same result as the library called from Python."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def harness(cuda_lib):
    if not O.ref_gpu_available():
        pytest.skip("reference harness builds not present (built from the reference sources by build())")
    return O


def _both(O, ic, periodic, **kw):
    args = dict(softening=tuple(ic["softening"]), dump=0, gt=1, **kw)
    if periodic:
        args.update(asmth=ic["asmth"], rcut=ic["rcut"])
    ref = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], periodic, **args)
    gpu = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], periodic, gpu=1, **args)
    return ref, gpu


@pytest.mark.parametrize("case", ["grid", "zoom"])
def test_gravity_step_bitexact_through_binding(harness, case):
    ic = ics.grid_box(n1=24, seed=41, pmgrid=48) if case == "grid" else ics.zoom_box(log2_half=14, seed=42, pmgrid=64)
    ref, gpu = _both(harness, ic, True)
    assert np.array_equal(ref["order_end"], gpu["order_end"])
    for ps in (0, 1):
        assert np.array_equal(ref[f"gacc{ps}"], gpu[f"gacc{ps}"]), ps
        assert np.array_equal(ref[f"oldacc{ps}"], gpu[f"oldacc{ps}"]), ps


def test_active_subset_through_binding(harness):
    ic = ics.zoom_box(log2_half=13, seed=43, pmgrid=64)
    ref, gpu = _both(harness, ic, True, active=7)
    act = np.arange(0, len(ic["mass"]), 7)
    for ps in (0, 1):
        assert np.array_equal(ref[f"gacc{ps}"][act], gpu[f"gacc{ps}"][act]), ps
        assert np.any(gpu[f"gacc{ps}"][act] != 0)


def test_out_of_box_recovery_through_binding(harness):
    ic = ics.hernquist(20000, seed=44)
    ref, gpu = _both(harness, ic, False, displace=0.3)
    assert "recoveries=1" in gpu["stdout"]
    assert np.array_equal(ref["order_end"], gpu["order_end"])  # both redid the domain decomposition
    for ps in (0, 1):
        assert np.array_equal(ref[f"gacc{ps}"], gpu[f"gacc{ps}"]), ps


def test_fp32_binding_matches_python_api(harness):
    ic = ics.zoom_box(log2_half=14, seed=45, pmgrid=64)
    r = harness.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"],
                        softening=tuple(ic["softening"]), dump=0, gt=1, gpu=2)
    with GravityTree(ics.params_for(ic, precision=L.PREC_FP32)) as t:
        acc, _, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
    order = r["order_end"]
    assert np.array_equal(r["gacc1"], acc[order])
