"""Gravity time steps and time bins on the GPU (gpugrav_timestep_gravity, gpugrav_active_particles):
get_timestep_gravity (src/time_integration/timestep.c:284-353) and the bin of
timebins_get_bin_and_do_validity_checks (timestep.c:725-770) per particle, bit-exact with the C oracle
(pinned to the reference's own functions by the CPU tests) and, where it is built, with the reference
harness itself; then the active list of the synchronized bins, which feeds gpugrav_walk_targets."""
import numpy as np
import pytest

from arepo_b200 import _lib as L
from arepo_b200 import ics
from arepo_b200.gravity import GravityTree
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TS = dict(eta=0.025, dtmax=0.01, dtmin=0.0, dtdisp=0.004)


def _tp(timebase=1 << 29, ti_current=0, sync=None, dtmin=0.0, nostop=False):
    tp = L.TimestepParams()
    tp.err_tol_int_accuracy = TS["eta"]
    tp.cf_atime = tp.cf_a2inv = tp.cf_hubble_a = 1.0
    tp.max_size_timestep, tp.min_size_timestep, tp.dt_displacement = TS["dtmax"], dtmin, TS["dtdisp"]
    tp.timebase_interval = 1.0 / timebase
    tp.timebase, tp.ti_current, tp.nostop_below_min = timebase, ti_current, int(nostop)
    for b in range(64):
        tp.synchronized[b] = 1 if (sync is None or sync[b]) else 0
    return tp


def test_timesteps_and_bins_bitexact(cuda_lib):
    ic = ics.zoom_box(log2_half=12, seed=71, pmgrid=64)
    soft = tuple(ic["softening"])
    prm = ics.params_for(ic)
    with GravityTree(prm) as t:
        acc, _, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        order = t.order()
        rng = np.random.default_rng(3)
        pm = 0.3 * acc * rng.normal(size=acc.shape)  # a stand-in long-range force
        bo = rng.integers(10, 25, len(acc)).astype(np.int8)
        sync = [b % 3 != 0 for b in range(64)]
        ti, bn = t.timestep_gravity(_tp(sync=sync), acc, ic["mass"], ic["softtype"], bo, grav_pm=pm)
    op = O.make_params(True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft)
    ti_o, bn_o, s = O.timestep_gravity(acc, ic["mass"], ic["softtype"], op, TS["eta"], TS["dtmax"], dtdisp=TS["dtdisp"],
                                       bin_old=bo, sync=sync, pm=pm)
    assert s == 0
    assert np.array_equal(ti, ti_o) and np.array_equal(bn, bn_o)
    assert len(np.unique(bn)) > 2  # several bins in use
    if O.ref_available():
        r = O.run_ref(ic["pos"], ic["mass"], ic["softtype"], True, asmth=ic["asmth"], rcut=ic["rcut"], softening=soft, dump=0,
                      gt=1, tstep=TS)
        o = r["order_end"]
        with GravityTree(prm) as t:
            ti_r, bn_r = t.timestep_gravity(_tp(), r["gacc1"], ic["mass"][o], ic["softtype"][o], np.zeros(len(o), np.int8))
        assert np.array_equal(ti_r, r["tistep"]) and np.array_equal(bn_r.astype(np.int32), r["tbin"])


def test_active_list_feeds_the_walk(cuda_lib):
    ic = ics.zoom_box(log2_half=12, seed=72, pmgrid=64)
    prm = ics.params_for(ic)
    with GravityTree(prm) as t:
        acc, _, _, oldacc = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        ti, bn = t.timestep_gravity(_tp(), acc, ic["mass"], ic["softtype"], np.zeros(len(acc), np.int8))
        top = int(np.median(bn))
        sync = [b <= top for b in range(64)]  # the bins that end now
        act = t.active_particles(bn, sync)
        assert np.array_equal(act, np.flatnonzero(bn <= top))
        prm.err_tol_theta = 0.0
        t.set_params(prm)
        a_act, _, _ = t.gravity_tree_targets(act, oldacc)
    assert np.array_equal(a_act, acc[act])  # the FP64 walk of the active subset = the full walk's rows


def test_timestep_errors(cuda_lib):
    ic = ics.hernquist(4096, seed=73)
    with GravityTree(ics.params_for(ic)) as t:
        acc, _, _, _ = t.compute_grav_accelerations(ic["pos"], ic["mass"], ic["softtype"])
        bo = np.zeros(len(acc), np.int8)
        with pytest.raises(L.GpuGravError) as e:  # the reference stops below MinSizeTimestep
            t.timestep_gravity(_tp(dtmin=1.0), acc, ic["mass"], ic["softtype"], bo)
        assert e.value.status == L.ERR_INVALID
        ti, bn = t.timestep_gravity(_tp(dtmin=1e-3, nostop=True), acc, ic["mass"], ic["softtype"], bo)
        assert np.all(ti >= int(1e-3 * (1 << 29)) - 1)
        ti, bn = t.timestep_gravity(_tp(ti_current=1 << 29), acc, ic["mass"], ic["softtype"], bo)
        assert np.all(bn == 0)  # end of the timeline
