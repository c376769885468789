"""Target slices (gpugrav_set_target_slice), the per-rank work of the sharded multi-GPU force
computation: for G slices the outputs of the G walks sum to the unsliced walk bit for bit (every
target is walked by exactly one slice, with the same tree and the same group, and the others
write zero), in both walk precisions, periodic and isolated."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree

pytestmark = pytest.mark.gpu

CASES = {
    "zoom": lambda: ics.zoom_box(log2_half=14, seed=1004, pmgrid=128),
    "plummer": lambda: ics.plummer(1 << 15, seed=8),
}


@pytest.mark.parametrize("precision", [L.PREC_FP32, L.PREC_FP64])
@pytest.mark.parametrize("name", list(CASES))
def test_slices_sum_to_unsliced_walk(name, precision, cuda_lib):
    ic = CASES[name]()
    prm = ics.params_for(ic, precision=precision)
    with GravityTree(prm) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        t.construct_forcetree()
        a_bh, _, _ = t.gravity_tree()
        oldacc = np.linalg.norm(a_bh, axis=1).astype(np.float32)
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        full_a, full_p, full_n = t.gravity_tree(oldacc)
        for g in (2, 3):
            sa, sp, sn = np.zeros_like(full_a), np.zeros_like(full_p), np.zeros_like(full_n)
            hit = np.zeros(len(full_n), np.int32)
            for s in range(g):
                t.set_target_slice(s, g)
                a, p, ni = t.gravity_tree(oldacc)
                sa += a
                sp += p
                sn += ni
                hit += (ni > 0)
            t.set_target_slice(0, 1)
            assert np.array_equal(sa, full_a)
            assert np.array_equal(sp, full_p)
            assert np.array_equal(sn, full_n)
            assert np.all(hit == 1)  # each target walked by exactly one slice
        with pytest.raises(L.GpuGravError):
            t.set_target_slice(3, 3)


@pytest.mark.parametrize("precision", [L.PREC_FP32, L.PREC_FP64])
def test_cost_balanced_slices_sum_to_unsliced_walk(precision, cuda_lib):
    """Slices of equal cost (the previous walk's interaction counts, as force_assign_cost_values):
    still every target exactly once and the sum bitwise the unsliced walk; the slices' interaction
    totals are far more even than with equal target counts on the zoom box."""
    ic = CASES["zoom"]()
    prm = ics.params_for(ic, precision=precision)
    g = 4
    with GravityTree(prm) as t:
        t.domain_decomposition(ic["pos"], ic["mass"], ic["softtype"])
        t.construct_forcetree()
        a_bh, _, _ = t.gravity_tree()
        oldacc = np.linalg.norm(a_bh, axis=1).astype(np.float32)
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        full_a, full_p, full_n = t.gravity_tree(oldacc)
        cost = full_n.astype(np.float32)
        sa, sp, sn = np.zeros_like(full_a), np.zeros_like(full_p), np.zeros_like(full_n)
        loads_cost, loads_count = [], []
        for s in range(g):
            t.set_target_slice_cost(s, g, cost)
            a, p, ni = t.gravity_tree(oldacc)
            sa += a
            sp += p
            sn += ni
            loads_cost.append(int(ni.sum()))
            t.set_target_slice(s, g)
            loads_count.append(int(t.gravity_tree(oldacc)[2].sum()))
        t.set_target_slice(0, 1)
    assert np.array_equal(sa, full_a) and np.array_equal(sp, full_p) and np.array_equal(sn, full_n)
    imb_cost = max(loads_cost) / np.mean(loads_cost)
    imb_count = max(loads_count) / np.mean(loads_count)
    assert imb_cost < 1.05 and imb_cost < imb_count, (loads_cost, loads_count)
