"""Benchmark of the short-range TreePM tree-gravity step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32] [--impl ours|reference]

Workload: the multi-mass zoom box, N = 2^24 (2^23 uniform low-resolution
particles of mass 8m plus 2^23 Plummer high-resolution particles of mass m, b =
0.02, truncated at 0.1), periodic, PMGRID = 512 (Asmth = 1.25/512, Rcut = 4.5
Asmth), two softening types (1/40 of the local mean spacing).  Seeded synthetic
particles (arepo_b200/ics.py).

One step = one short-range force computation with the relative opening
criterion, exactly what gravity() runs after the first step: Peano-Hilbert keys,
stable key sort, top-level tree, octree build with moments, tree walk for every
particle.  OldAcc comes from a Barnes-Hut pass done once before the warm-up.
`value` is particles per second with inputs resident in device memory; `e2e` is
the same metric through the C ABI with host buffers (uploads and downloads inside
the timed region).  Inputs (positions, tree, walk layout: > 2 GB) exceed the 126 MB
L2, so no flush is needed between steps.

With --gpus N (torchrun, one process per GPU) every rank runs its own
independent zoom box (seed + rank): replicas, weak scaling, no collective on
the data path; the step time is the maximum over ranks.

--impl reference times the reference's own C (oracle/_ref, compiled from the
reference sources) on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tree-gravity particles/s at N=2^24 (RMS force err ≤1e-3); serving p50/p99 latency"
UNIT = "particles/s"
FLOPS_PER_INTERACTION = 23.0  # convention of the path's roofline


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_config(log2_half, precision, alpha):
    return {
        "workload": f"zoom box N=2^{log2_half + 1}: 2^{log2_half} uniform (mass 8m) + 2^{log2_half} Plummer b=0.02 r<0.1 "
                    f"(mass m), periodic L=1, PMGRID=512, RCUT=4.5, ASMTH=1.25, 2 softening types, relative criterion "
                    f"ErrTolForceAcc={alpha} after a Barnes-Hut pass (theta=0.7)",
        "err_tol_force_acc": alpha,
        "n_particles": 1 << (log2_half + 1),
        "step": "keys+sort+toptree+build+moments+walk (all particles are targets)",
        "walk_precision": precision,
        "l2": "inputs larger than L2 (no flush)",
        "global_batch": 1 << (log2_half + 1),
        "parallelism": "replicas",
    }


# --------------------------------------------------------------------------------------
# clocks during the timed region (NVML reads only)
# --------------------------------------------------------------------------------------
class ClockSampler:
    REASONS = {
        "gpu_idle": 0x1,
        "applications_clocks_setting": 0x2,
        "sw_power_cap": 0x4,
        "hw_slowdown": 0x8,
        "sync_boost": 0x10,
        "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index):
        self.samples, self.reasons, self.ok = [], set(), False
        self.stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # no NVML: report nothing rather than guess
            log("clock sampling unavailable:", e)
            self.max_mhz = None

    def _run(self):
        while not self.stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for k, v in self.REASONS.items():
                    if r & v and k != "gpu_idle":
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(0.1)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.ok:
            self.t.join()

    def report(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons)}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# --------------------------------------------------------------------------------------
# CPU reference (oracle/_ref: the reference's own compiled code)
# --------------------------------------------------------------------------------------
CPU_SAMPLE_LOG2_HALF = 19   # N = 2^20 particles of the same zoom distribution
CPU_SAMPLE_STRIDE = 64      # walk every 64th target, extrapolated to all


def run_cpu_reference(procs: int, alpha: float, log2_half: int = CPU_SAMPLE_LOG2_HALF, stride: int = CPU_SAMPLE_STRIDE):
    """Reference step on the host: domain decomposition (keys, sort, top tree), construct_forcetree,
    force_treeevaluate for a 1/stride sample of targets after a Barnes-Hut pass, by `procs` independent
    processes that each walk a disjoint slice of the sample. Returns (particles/s, detail)."""
    from arepo_b200 import ics
    from oracle import oracle as O

    exe = os.path.join(O.REF_DIR, "ref_harness_pm")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    ic = ics.zoom_box(log2_half=log2_half, seed=1004, pmgrid=512)
    n = len(ic["mass"])
    import tempfile

    td = tempfile.mkdtemp()
    fin = os.path.join(td, "in.bin")
    O.write_input(fin, ic["pos"], ic["mass"], ic["softtype"])
    eps = ic["softening"]
    slice_len = (n + procs - 1) // procs
    ps = []
    for p in range(procs):
        fout = os.path.join(td, f"out{p}.bin")
        args = [exe, fin, fout, "box=1.0", f"asmth={ic['asmth']!r}", f"rcut={ic['rcut']!r}", "theta=0.7",
                f"erracc={alpha!r}", f"eps0={eps[0]!r}", f"eps1={eps[1]!r}", "mdom=8", "tnf=2.5", "passes=2", "dump=0",
                "gt=0", f"stride={stride}", f"first={p * slice_len}", f"count={min(slice_len, n - p * slice_len)}"]
        ps.append((subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.PIPE), fout))
    times = []
    for proc, fout in ps:
        proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError("reference harness failed")
        r = O.read_output(fout)
        times.append(r["time1"])  # relative pass: domain, build, walk(sample), -, targets, interactions
    t = np.array(times)
    domain, build = t[:, 0].max(), t[:, 1].max()
    walk_full = (t[:, 2] * stride).max()  # each process walks its slice; extrapolate the 1/stride sample
    step = domain + build + walk_full
    ia = t[:, 5].sum() * stride
    detail = {"n": n, "procs": procs, "domain_s": domain, "build_s": build, "walk_s_extrapolated": walk_full,
              "interactions_per_particle": ia / n}
    return n / step, detail


def cpu_info():
    try:
        model = [l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name")][0]
    except Exception:
        model = "unknown"
    return model, os.cpu_count()


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    model, ncpu = cpu_info()
    procs = max(1, min(ncpu or 1, 16))
    vals = []
    for k in range(args.warmup + args.steps):
        v, detail = run_cpu_reference(procs, args.err_tol_force_acc)
        if k >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * detail["n"] / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(23, "fp64", args.err_tol_force_acc), cpu_sample=f"N=2^{CPU_SAMPLE_LOG2_HALF + 1} of the same zoom "
                       f"distribution, 1/{CPU_SAMPLE_STRIDE} of targets walked and extrapolated"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": f"reference C (oracle/_ref), {procs} processes on {model}; N=2^{CPU_SAMPLE_LOG2_HALF + 1} "
                                   f"zoom box, domain+build+walk, walk on 1/{CPU_SAMPLE_STRIDE} targets extrapolated",
                         "detail": detail},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------
def our_arm(args):
    import torch

    from arepo_b200 import _lib as L
    from arepo_b200 import ics
    from arepo_b200.gravity import GravityTree

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        log(f"warning: --gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()

    prec = L.PREC_FP32 if args.precision == "fp32" else L.PREC_FP64
    lh = args.log2_half
    t0 = time.time()
    ic = ics.zoom_box(log2_half=lh, seed=1004 + rank, pmgrid=512)
    n = len(ic["mass"])
    log(f"rank {rank}: generated N={n} in {time.time() - t0:.1f}s")
    dev = torch.device("cuda", local)
    pos_d = torch.from_numpy(ic["pos"]).to(dev)
    mass_d = torch.from_numpy(ic["mass"]).to(dev)
    st_d = torch.from_numpy(ic["softtype"]).to(dev)
    acc_d = torch.empty((n, 3), dtype=torch.float64, device=dev)
    pot_d = torch.empty(n, dtype=torch.float64, device=dev)
    ni_d = torch.empty(n, dtype=torch.int32, device=dev)

    prm = ics.params_for(ic, precision=prec)
    tree = GravityTree(prm, device=local)
    stream = torch.cuda.Stream(device=dev)
    tree.set_stream(stream.cuda_stream)
    lib = tree.lib
    ctx = tree._ctx

    def compute(oldacc_ptr, mem, pos, mass, st, acc, pot, ni):
        s = lib.gpugrav_compute(ctx, n, L.ptr(pos), L.ptr(mass), L.ptr(st), oldacc_ptr, None, None, 0, L.ptr(acc),
                                L.ptr(pot), L.ptr(ni), mem)
        if s != 0:
            raise L.GpuGravError(s, lib.gpugrav_last_error(ctx).decode())

    # Barnes-Hut pass (first step) -> OldAcc
    compute(None, L.MEM_DEVICE, pos_d, mass_d, st_d, acc_d, pot_d, ni_d)
    oldacc_d = torch.linalg.norm(acc_d, dim=1).to(torch.float32)
    prm.err_tol_theta = 0.0
    prm.err_tol_force_acc = args.err_tol_force_acc
    tree.set_params(prm)
    info = None

    # warm-up (relative criterion)
    for _ in range(args.warmup):
        compute(L.ptr(oldacc_d), L.MEM_DEVICE, pos_d, mass_d, st_d, acc_d, pot_d, ni_d)
    info = tree.tree_info()
    torch.cuda.synchronize()

    # ---- timed: device-resident inputs ----
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    walk_ms, build_ms, domain_ms, sort_ms, inter = [], [], [], [], []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            compute(L.ptr(oldacc_d), L.MEM_DEVICE, pos_d, mass_d, st_d, acc_d, pot_d, ni_d)
            tm = tree.timings()
            walk_ms.append(tm.walk_ms)
            build_ms.append(tm.build_ms + tm.toptree_ms)
            domain_ms.append(tm.domain_ms)
            sort_ms.append(tm.sort_ms)
            inter.append(tm.interactions)
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end) / args.steps
    launches_per_step = 5 + tm.build_kernel_launches + 3  # extent x2, keys, gather, (sort: CUB) ; build ; walk gather/walk/scatter
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # ---- timed: host buffers through the C ABI (end to end) ----
    pos_h = torch.from_numpy(ic["pos"]).pin_memory()
    mass_h = torch.from_numpy(ic["mass"]).pin_memory()
    st_h = torch.from_numpy(ic["softtype"]).pin_memory()
    old_h = oldacc_d.cpu().pin_memory()
    acc_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    pot_h = torch.empty(n, dtype=torch.float64).pin_memory()
    ni_h = torch.empty(n, dtype=torch.int32).pin_memory()
    compute(L.ptr(old_h), L.MEM_HOST, pos_h, mass_h, st_h, acc_h, pot_h, ni_h)
    barrier()
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        compute(L.ptr(old_h), L.MEM_HOST, pos_h, mass_h, st_h, acc_h, pot_h, ni_h)
    end.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = start.elapsed_time(end) / args.steps
    if dist is not None:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())

    # ---- accuracy against FP64 direct summation on 8192 sampled targets ----
    rng = np.random.default_rng(2004)
    tg = np.sort(rng.choice(n, 8192, replace=False))
    acc_tree = acc_h.numpy()[tg]

    def err_stats(acc_dir):
        dn = np.linalg.norm(acc_dir, axis=1)
        err_abs = np.linalg.norm(acc_tree - acc_dir, axis=1)
        rel = err_abs / np.maximum(dn, 1e-300)
        rms_force = np.sqrt(np.mean(dn * dn))
        return {"rms_rel": float(np.sqrt(np.mean(rel * rel))), "p99_rel": float(np.percentile(rel, 99)),
                "median_rel": float(np.median(rel)),
                "rms_rel_to_rms_force": float(np.sqrt(np.mean((err_abs / rms_force) ** 2)))}

    acc_cut, _ = tree.direct(tg, cut=True)
    acc_full, _ = tree.direct(tg, cut=False)
    acc_stats = dict(err_stats(acc_cut), targets=int(len(tg)),
                     reference="FP64 direct sum over pairs closer than Rcut with the exact erfc factor (the range the "
                               "walk evaluates): the tree approximation error",
                     vs_full_short_range=err_stats(acc_full))

    # ---- roofline of the walk kernel (device time measured with CUDA events on its stream) ----
    pk = L.C.c_double(0.0)
    lib.gpugrav_measure_fma_peak(local, prec, L.C.byref(pk))
    peak = float(pk.value)
    walk_s = float(np.mean(walk_ms)) * 1e-3
    ia = float(np.mean(inter))
    achieved = FLOPS_PER_INTERACTION * ia / walk_s / 1e12
    roofline = {"bound": "fp32" if prec == L.PREC_FP32 else "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None, "traffic": None,
                "kernel": "k_walk32" if prec == L.PREC_FP32 else "k_walk64",
                "peak_source": "measured in-run: CUDA-core FMA microbenchmark (gpugrav_measure_fma_peak); "
                               "MEASURED_PEAKS.json has no CUDA-core figure",
                "flops_per_interaction": FLOPS_PER_INTERACTION, "interactions_per_step": ia,
                "walk_ms": float(np.mean(walk_ms)), "build_ms": float(np.mean(build_ms)),
                "domain_ms": float(np.mean(domain_ms)), "sort_ms": float(np.mean(sort_ms))}

    value = world * n / (ms * 1e-3)
    e2e_value = world * n / (ms_e2e * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == L.PREC_FP32 else "f64", "data": "synthetic (seeded zoom box, arepo_b200/ics.py)",
        "config": workload_config(lh, args.precision, args.err_tol_force_acc),
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": ms_e2e, "h2d_bytes_per_step": n * (24 + 8 + 1 + 4),
                "d2h_bytes_per_step": n * (24 + 8 + 4)},
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clk.report(),
        "accuracy": acc_stats,
        "interactions_per_particle": ia / n,
        "tree": {"num_nodes": int(info.num_nodes), "max_depth": int(info.max_depth),
                 "topnodes": int(info.num_topnodes)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            model, ncpu = cpu_info()
            v, detail = run_cpu_reference(1, args.err_tol_force_acc)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"reference C (oracle/_ref) on 1 core of {model}: N=2^{CPU_SAMPLE_LOG2_HALF + 1} "
                                              f"zoom box, domain+build+walk, walk on 1/{CPU_SAMPLE_STRIDE} targets extrapolated",
                                    "detail": detail}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    tree.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--err-tol-force-acc", type=float, default=5e-5,
                    help="ErrTolForceAcc of the timed relative-criterion steps; 5e-5 keeps the FP32 walk's RMS force "
                         "error below 1e-3 on the zoom box (the metric's accuracy bar)")
    ap.add_argument("--log2-half", type=int, default=23, help="log2 of each species' count (23 -> N=2^24)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
