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

With --gpus N (torchrun, one process per GPU) the same zoom box (N = 2^24 in
total) is sharded: every rank owns 1/N of the particles, a step all-gathers the
particles over NCCL, builds the same tree on every GPU, walks the rank's own
key-ordered slice of the targets and reduce-scatters the forces to their owners
(arepo_b200/sharded.py).  Total work is fixed: strong scaling; the step time is
the maximum over ranks.

Serving leg (rank 0 at N=1; --no-serving skips it): a seeded stream of isolated
systems (Plummer spheres and Hernquist haloes, 50/50, N log-uniform in
[10^3, 10^6], G=1, softening 0.02 scale radius, FP32 walk, ErrTolForceAcc 0.0025),
each running the first-step sequence (Barnes-Hut pass, relative pass) and K=16
kick-drift-kick steps of dt=0.005 under a 120 GB admission budget.  Throughput
(requests/s, particle-steps/s) all-arrived-at-once for the continuously batched
server and for one-request-at-a-time execution (max_systems=1) on the same
requests; p50/p99 latency under Poisson arrivals at a fraction of the batched
capacity.  Wall clock of the host-driven serving loop: admission uploads, every
tick's kernels and result downloads are inside it.  --serve-requests 10000 runs
the full stream.

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
# DRAM bytes (read + write) of one FP32 walk launch per particle: ncu capture of the zoom box at
# N=2^21 (dram__bytes_read.sum + dram__bytes_write.sum = 298.9 MB + 84.3 MB), scaled by the
# particle count (the walk reads the tree and the particles once from DRAM; everything else hits
# in L2)
WALK32_DRAM_BYTES_PER_PARTICLE = 383.2e6 / (1 << 21)
# ErrTolForceAcc of the per-target FP64 walk in the precision ablation: the value at which its RMS
# error on the zoom box is at most the FP32 walk's at 6e-5 (8.2e-4 against 9.4e-4)
ABLATION_FP64_ALPHA = 2e-5


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_config(log2_half, precision, alpha, world=1):
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
        "parallelism": "one GPU" if world == 1 else
                       f"one system sharded over {world} GPUs: all-gather of particles (NCCL), identical trees, "
                       f"one key-ordered target slice per GPU, reduce-scatter of forces",
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
CPU_LOG2_HALF = 23        # the GPU arm's zoom box: N = 2^24
CPU_SAMPLE_STRIDE = 1024  # every 1024th target of the zoom box (16384 of 2^24) per timed walk


def run_cpu_reference(procs: int, alpha: float, reps: int, log2_half: int | None = None, stride: int | None = None):
    """The reference's own code (oracle/_ref/ref_harness_pm, compiled from the reference sources) on the
    same particles as the GPU arm: domain_Decomposition and construct_forcetree of every particle (timed
    once), force_treeevaluate for every stride-th target in key order in a Barnes-Hut pass (OldAcc) and a
    relative pass, then `reps` more timed walks of that sample by `procs` forked processes that share the
    particles and the tree.  Each target's walk is independent, so the walk of all targets takes
    (walk of the sample) x (targets / sample).  Returns a dict of the measured figures."""
    from arepo_b200 import ics
    from oracle import oracle as O

    stride = CPU_SAMPLE_STRIDE if stride is None else stride
    log2_half = CPU_LOG2_HALF if log2_half is None else log2_half
    exe = os.path.join(O.REF_DIR, "ref_harness_pm")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    ic = ics.zoom_box(log2_half=log2_half, seed=1004, pmgrid=512)
    n = len(ic["mass"])
    import tempfile

    td = tempfile.mkdtemp()
    fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
    O.write_input(fin, ic["pos"], ic["mass"], ic["softtype"])
    del ic
    eps = ics.zoom_box_softening(log2_half)
    a = ics.ASMTH / 512
    args = [exe, fin, fout, "box=1.0", f"asmth={a!r}", f"rcut={ics.RCUT * a!r}", "theta=0.7", f"erracc={alpha!r}",
            f"eps0={eps[0]!r}", f"eps1={eps[1]!r}", "mdom=8", "tnf=2.5", "passes=2", "dump=0", "gt=0", "lite=1",
            f"stride={stride}", f"procs={procs}", f"reps={reps}"]
    t0 = time.time()
    r = subprocess.run(args, capture_output=True, text=True)
    wall = time.time() - t0
    for f in (fin, fout):
        if os.path.exists(f):
            os.remove(f)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-500:]}")

    def fields(line):
        return {k: v for k, v in (w.split("=", 1) for w in line.replace("(", "").replace(")", "").replace(",", "").split()
                                   if "=" in w)}

    passes = [fields(l) for l in r.stdout.splitlines() if l.startswith("pass=")]
    reps_ = [fields(l) for l in r.stdout.splitlines() if l.startswith("rep=")]
    if len(passes) != 2 or len(reps_) != reps:
        raise RuntimeError("unexpected reference harness output")
    targets = int(reps_[0]["targets"])
    return {"n": n, "targets": targets, "stride": stride, "procs": procs,
            "domain_s": float(passes[0]["domain"]), "build_s": float(passes[1]["build"]),
            "walk_s": [float(x["walk"]) for x in reps_],
            "interactions_per_target": int(reps_[0]["interactions"]) / targets, "harness_wall_s": wall}


def cpu_reference_value(d, walk_s):
    """particles/s of one full step (domain decomposition + tree build + walk of every particle) from the
    measured set-up and the walk of the sample, extrapolated linearly in the number of targets"""
    step = d["domain_s"] + d["build_s"] + walk_s * d["n"] / d["targets"]
    return d["n"] / step, step


def cpu_info():
    try:
        model = [l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name")][0]
    except Exception:
        model = "unknown"
    return model, os.cpu_count()


def cpu_sample_text(d, model):
    return (f"reference C (oracle/_ref, the reference's own sources), {d['procs']} forked processes on {model}: the same "
            f"N=2^{int(d['n']).bit_length() - 1} zoom box and ErrTolForceAcc; domain decomposition + tree build of all particles measured once "
            f"({d['domain_s']:.1f} s + {d['build_s']:.1f} s); each step walks every {d['stride']}th target in key order "
            f"({d['targets']} targets, {d['interactions_per_target']:.0f} interactions each); full-step particles/s "
            f"= N / (set-up + sample walk x N/{d['targets']})")


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    model, ncpu = cpu_info()
    procs = max(1, ncpu or 1)
    d = run_cpu_reference(procs, args.err_tol_force_acc, args.warmup + args.steps)
    timed = d["walk_s"][args.warmup:]
    vals = [cpu_reference_value(d, w)[0] for w in timed]
    value = float(np.mean(vals))
    ms = 1e3 * float(np.mean(timed))
    detail = dict(d, walk_s=None, walk_s_timed=timed, full_step_s_extrapolated=cpu_reference_value(d, float(np.mean(timed)))[1])
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded zoom box, arepo_b200/ics.py)",
        "config": dict(workload_config(CPU_LOG2_HALF, "fp64", args.err_tol_force_acc),
                       step="one timed step = the walk of the sample (every "
                            f"{d['stride']}th target) by {procs} processes; value = full-step particles/s "
                            "(measured domain decomposition and build + sample walk scaled to all targets)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": cpu_sample_text(d, model), "detail": detail},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
# serving leg
# --------------------------------------------------------------------------------------
SERVE_NMIN, SERVE_NMAX = 1000, 1000000
SERVE_EPS, SERVE_K, SERVE_DT = 0.02, 16, 0.005
SERVE_BUDGET = 120e9
SERVE_CLASS_REQUESTS = 16  # requests per size decade in the per-class comparison


def serving_stream(count: int, seed: int = 1005):
    """Sizes (log-uniform in [SERVE_NMIN, SERVE_NMAX]) and kinds (0 Plummer, 1 Hernquist) of the stream."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(SERVE_NMIN), np.log(SERVE_NMAX), count)).astype(np.int64)
    return ns, rng.integers(0, 2, count)


def serving_system(n: int, kind: int, seed: int):
    from arepo_b200 import ics

    ic = ics.plummer(n, seed, eps=SERVE_EPS) if kind == 0 else ics.hernquist(n, seed=seed, eps=SERVE_EPS)
    return ic["pos"], np.zeros_like(ic["pos"]), ic["mass"], ic["softtype"]


def run_stream(systems, ids, arrivals, max_systems, device, max_particles):
    """Serve requests `ids` (arrival offsets in seconds, or None: all at once) and return throughput
    and latency figures. Latency runs from the scheduled arrival to the poll that returned the result."""
    from arepo_b200.serving import GravityServer, serving_params

    prm = serving_params(SERVE_EPS)
    warm = serving_system(2000, 0, 99)
    with GravityServer(prm, device=device, max_systems=max_systems, max_particles=max_particles,
                       budget_bytes=SERVE_BUDGET) as srv:
        for w in range(2):  # warm-up: first buffers, graph capture
            srv.submit((1 << 40) + w, *warm, nsteps=1, dt=SERVE_DT)
        srv.run_to_completion()
        s0 = srv.stats()
        arrive, lat, svc, sizes = {}, [], [], []
        # result buffers allocated (and touched) before the timed region, as a serving client would
        # (up to 8 GB of them; beyond, each result gets new arrays when it is polled)
        nres = sum(len(systems[int(i)][2]) for i in ids)
        outbufs = None
        if nres * 72 <= 8e9:
            outbufs = {int(i): tuple(np.full((len(systems[int(i)][2]), 3), 0.0) for _ in range(3)) for i in ids}
        k, nsys_ticks = 0, 0
        t_sub = t_poll = 0.0
        t0 = time.monotonic()
        while True:
            now = time.monotonic() - t0
            while k < len(ids) and (arrivals is None or arrivals[k] <= now):
                i = int(ids[k])
                arrive[i] = t0 + (0.0 if arrivals is None else float(arrivals[k]))
                ts = time.monotonic()
                srv.submit(i, *systems[i], nsteps=SERVE_K, dt=SERVE_DT)
                t_sub += time.monotonic() - ts
                k += 1
            if not srv.busy():
                if k >= len(ids):
                    break
                time.sleep(max(0.0, float(arrivals[k]) - (time.monotonic() - t0)))
                continue
            srv.tick()
            nsys_ticks += srv.stats().last_tick_systems
            tp = time.monotonic()
            for r in srv.poll_all(outbufs):
                lat.append(time.monotonic() - arrive[r.id])
                svc.append(r.t_done - r.t_admit)
                sizes.append(len(r.pos))
            t_poll += time.monotonic() - tp
        wall = time.monotonic() - t0
        s1 = srv.stats()
    ticks = s1.ticks - s0.ticks
    return {"requests": len(ids), "wall_s": wall, "requests_per_s": len(ids) / wall,
            "particle_steps_per_s": (s1.particle_steps - s0.particle_steps) / wall,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "service_p50_s": float(np.percentile(svc, 50)), "service_p99_s": float(np.percentile(svc, 99)),
            "ticks": int(ticks), "mean_systems_per_tick": nsys_ticks / max(ticks, 1),
            "phase_s": dict({k: getattr(s1, k) - getattr(s0, k)
                             for k in ("admit_s", "build_s", "keys_s", "tree_s", "walk_s", "finish_s")},
                            submit_s=t_sub, poll_s=t_poll),
            "interactions_per_particle_step": (s1.interactions - s0.interactions) / max(1, s1.particle_steps - s0.particle_steps),
            "graph_captures": int(s1.graph_captures - s0.graph_captures),
            "graph_replays": int(s1.graph_replays - s0.graph_replays)}


def run_plain_serial(systems, ids, device):
    """The same requests one at a time through the plain per-call API: one gpugrav_compute per force
    evaluation on host arrays (upload, keys, sort, build, walk, download), kick and drift on the host
    -- the pattern of a code that calls gravity once per step."""
    from arepo_b200 import _lib as L
    from arepo_b200.gravity import GravityTree
    from arepo_b200.serving import serving_params

    prm = serving_params(SERVE_EPS)
    theta = prm.err_tol_theta
    lat, steps = [], 0
    with GravityTree(prm, device=device) as t:
        lib, ctx = t.lib, t._ctx

        def force(x, mass, st, old):
            n = len(mass)
            acc = np.empty((n, 3))
            ni = np.empty(n, np.int32)
            s = lib.gpugrav_compute(ctx, n, L.ptr(x), L.ptr(mass), L.ptr(st), None if old is None else L.ptr(old), None,
                                    None, 0, L.ptr(acc), None, L.ptr(ni), L.MEM_HOST)
            if s != 0:
                raise L.GpuGravError(s, lib.gpugrav_last_error(ctx).decode())
            return acc

        def run(i):
            pos, vel, mass, st = systems[i]
            x, v = pos.copy(), vel.copy()
            prm.err_tol_theta = theta
            t.set_params(prm)
            a = force(x, mass, st, None)  # Barnes-Hut pass
            prm.err_tol_theta = 0.0
            t.set_params(prm)
            a = force(x, mass, st, np.linalg.norm(a, axis=1).astype(np.float32))  # relative pass
            for _ in range(SERVE_K):
                v += 0.5 * SERVE_DT * a
                x += SERVE_DT * v
                a = force(x, mass, st, np.linalg.norm(a, axis=1).astype(np.float32))
                v += 0.5 * SERVE_DT * a
            return (SERVE_K + 2) * len(mass)

        run(int(ids[0]))  # warm-up
        t0 = time.monotonic()
        for i in ids:
            steps += run(int(i))
            lat.append(time.monotonic() - t0)
        wall = time.monotonic() - t0
    return {"requests": len(ids), "wall_s": wall, "requests_per_s": len(ids) / wall, "particle_steps_per_s": steps / wall,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99))}


def serving_leg(args, device):
    ns, kinds = serving_stream(args.serve_requests)
    t = time.time()
    systems = [serving_system(int(ns[i]), int(kinds[i]), 5000 + i) for i in range(len(ns))]
    log(f"serving: generated {len(ns)} systems ({int(ns.sum())} particles) in {time.time() - t:.1f}s")
    pool = int(min(1 << 27, max(int(ns.sum()), SERVE_NMAX) + 4096))
    ncmp = min(args.serve_compare, len(ns))
    cmp_ids = np.arange(ncmp)
    batched = run_stream(systems, cmp_ids, None, 4096, device, pool)
    log(f"serving: batched {batched['requests_per_s']:.2f} req/s")
    serial = run_stream(systems, cmp_ids, None, 1, device, pool)
    log(f"serving: serial {serial['requests_per_s']:.2f} req/s")
    plain = run_plain_serial(systems, cmp_ids, device)
    log(f"serving: plain API serial {plain['requests_per_s']:.2f} req/s")
    # the same comparison per decade of system size: where continuous batching pays
    by_size = []
    for lo_n, hi_n in ((SERVE_NMIN, 10 * SERVE_NMIN), (10 * SERVE_NMIN, 100 * SERVE_NMIN), (100 * SERVE_NMIN, SERVE_NMAX + 1)):
        ids = np.nonzero((ns >= lo_n) & (ns < hi_n))[0][:SERVE_CLASS_REQUESTS]
        if len(ids) == 0:
            continue
        b = run_stream(systems, ids, None, 4096, device, pool)
        s1 = run_stream(systems, ids, None, 1, device, pool)
        by_size.append({"n_range": [int(lo_n), int(hi_n)], "requests": int(len(ids)),
                        "particles": int(ns[ids].sum()),
                        "batched_requests_per_s": b["requests_per_s"], "serial_requests_per_s": s1["requests_per_s"],
                        "batched_particle_steps_per_s": b["particle_steps_per_s"],
                        "serial_particle_steps_per_s": s1["particle_steps_per_s"],
                        "batched_latency_p99_s": b["latency_p99_s"], "serial_latency_p99_s": s1["latency_p99_s"],
                        "throughput_ratio": b["particle_steps_per_s"] / s1["particle_steps_per_s"]})
        log(f"serving: N in [{lo_n}, {hi_n}): batched/serial {by_size[-1]['throughput_ratio']:.2f}")
    rate = args.serve_load * batched["requests_per_s"]
    arr = np.cumsum(np.random.default_rng(1006).exponential(1.0 / rate, len(ns)))
    poisson = run_stream(systems, np.arange(len(ns)), arr, 4096, device, pool)
    log(f"serving: poisson p50 {poisson['latency_p50_s']:.2f}s p99 {poisson['latency_p99_s']:.2f}s")
    return {
        "stream": f"{len(ns)} isolated systems, Plummer/Hernquist 50/50 (seeded), N log-uniform in "
                  f"[{SERVE_NMIN}, {SERVE_NMAX}], G=1, softening {SERVE_EPS} scale radius, zero initial velocities, "
                  f"BH pass + relative pass (ErrTolForceAcc 0.0025) + K={SERVE_K} KDK steps of dt={SERVE_DT}, "
                  f"FP32 walk, {SERVE_BUDGET / 1e9:.0f} GB admission budget",
        "particles": int(ns.sum()),
        "compare": {"requests": int(ncmp), "arrivals": "all at t=0", "batched": batched,
                    "serial_max_systems_1": serial, "serial_plain_api": plain,
                    "throughput_ratio": batched["particle_steps_per_s"] / serial["particle_steps_per_s"],
                    "throughput_ratio_vs_plain_api": batched["particle_steps_per_s"] / plain["particle_steps_per_s"],
                    "serial_note": "serial_max_systems_1: the serving loop admitting one request at a time (device-"
                                   "resident particles, the same kernels); serial_plain_api: one gpugrav_compute call "
                                   "per force evaluation on host arrays, kick/drift on the host"},
        "by_size_class": by_size,
        "poisson": dict(poisson, rate_per_s=rate, load=args.serve_load),
        "clock": "host wall clock of the serving loop (uploads, ticks, downloads included)",
    }


# --------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------
def sharded_arm(args):
    """N > 1: one zoom box sharded over the ranks (see the module docstring)."""
    import datetime

    import torch
    import torch.distributed as dist

    from arepo_b200 import _lib as L
    from arepo_b200 import ics
    from arepo_b200.sharded import ShardedGravity

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # stdout carries the JSON line only: what the libraries print (NCCL's version banner) goes to stderr
    sys.stdout.flush()
    stdout_fd = os.dup(1)
    os.dup2(2, 1)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29541")
    os.environ.setdefault("RANK", str(rank))
    os.environ.setdefault("WORLD_SIZE", str(world))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    prec = L.PREC_FP32 if args.precision == "fp32" else L.PREC_FP64
    lh = args.log2_half
    ic = ics.zoom_box(log2_half=lh, seed=1004, pmgrid=512)
    n = len(ic["mass"])
    lo, hi = n * rank // world, n * (rank + 1) // world
    pos_h = torch.from_numpy(ic["pos"][lo:hi].copy()).pin_memory()
    mass_h = torch.from_numpy(ic["mass"][lo:hi].copy()).pin_memory()
    st_h = torch.from_numpy(ic["softtype"][lo:hi].copy()).pin_memory()
    pos_d, mass_d, st_d = pos_h.to(dev), mass_h.to(dev), st_h.to(dev)
    prm = ics.params_for(ic, precision=prec)
    sg = ShardedGravity(prm, device=local)
    tree = sg._tree
    stream = torch.cuda.current_stream()

    acc_d, _, _ = sg.compute(pos_d, mass_d, st_d, None)  # Barnes-Hut pass -> OldAcc
    oldacc_d = torch.linalg.norm(acc_d, dim=1).to(torch.float32)
    prm.err_tol_theta = 0.0
    prm.err_tol_force_acc = args.err_tol_force_acc
    tree.set_params(prm)
    # slices of equal cost: each step's interaction counts balance the next step's slices
    cost_d = None
    for _ in range(args.warmup):
        acc_d, _, ni_d = sg.compute(pos_d, mass_d, st_d, oldacc_d, cost_d)
        cost_d = ni_d.to(torch.float32)
    torch.cuda.synchronize()

    def timed(fn):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            fn()
        end.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        t = torch.tensor([start.elapsed_time(end) / args.steps], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    walk_ms, inter = [], []

    def step():
        sg.compute(pos_d, mass_d, st_d, oldacc_d, cost_d)
        tm = tree.timings()
        walk_ms.append(tm.walk_ms)
        inter.append(tm.interactions)

    with ClockSampler(local) as clk:
        ms = timed(step)
    old_h = oldacc_d.cpu().pin_memory()
    acc_h = torch.empty((hi - lo, 3), dtype=torch.float64).pin_memory()

    def step_e2e():
        a, _, _ = sg.compute(pos_h.to(dev, non_blocking=True), mass_h.to(dev, non_blocking=True),
                             st_h.to(dev, non_blocking=True), old_h.to(dev, non_blocking=True), cost_d)
        acc_h.copy_(a, non_blocking=True)

    ms_e2e = timed(step_e2e)

    line = None
    if rank == 0:
        rng = np.random.default_rng(2004)
        tg = np.sort(rng.choice(hi - lo, min(8192, hi - lo), replace=False))
        acc_tree = acc_h.numpy()[tg]
        d_cut, _ = tree.direct(tg, cut=True)  # the tree context holds all particles, rank order = input order
        dn = np.linalg.norm(d_cut, axis=1)
        rel = np.linalg.norm(acc_tree - d_cut, axis=1) / np.maximum(dn, 1e-300)
        pk = L.C.c_double(0.0)
        tree.lib.gpugrav_measure_fma_peak(local, prec, L.C.byref(pk))
        peak = float(pk.value)
        walk_s = float(np.mean(walk_ms)) * 1e-3
        ia = float(np.mean(inter))
        achieved = FLOPS_PER_INTERACTION * ia / walk_s / 1e12
        line = {
            "metric": METRIC, "value": n / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if prec == L.PREC_FP32 else "f64", "data": "synthetic (seeded zoom box, arepo_b200/ics.py)",
            "config": workload_config(lh, args.precision, args.err_tol_force_acc, world),
            "roofline": {"bound": "fp32" if prec == L.PREC_FP32 else "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None,
                         "traffic": WALK32_DRAM_BYTES_PER_PARTICLE * n / world if prec == L.PREC_FP32 else None,
                         "kernel": "k_walk32" if prec == L.PREC_FP32 else "k_walk64",
                         "scope": "rank 0's walk of its target slice",
                         "walk_ms": float(np.mean(walk_ms)), "interactions_per_step": ia},
            "e2e": {"value": n / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": world * (hi - lo) * (24 + 8 + 1 + 4),
                    "d2h_bytes_per_step": world * (hi - lo) * 24},
            "gpu_launches": int((5 + tree.timings().build_kernel_launches + 4) * args.steps),
            "clocks": clk.report(),
            "accuracy": {"rms_rel": float(np.sqrt(np.mean(rel * rel))), "p99_rel": float(np.percentile(rel, 99)),
                         "targets": int(len(tg)), "reference": "FP64 direct sum over pairs closer than Rcut, rank 0's particles"},
        }
    sg.close()
    dist.barrier()
    dist.destroy_process_group()
    sys.stdout.flush()
    os.dup2(stdout_fd, 1)
    os.close(stdout_fd)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def our_arm(args):
    """One GPU, one process (more ranks run sharded_arm)."""
    import torch

    from arepo_b200 import _lib as L
    from arepo_b200 import ics
    from arepo_b200.gravity import GravityTree

    world, rank, local = 1, 0, int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != 1:
        log(f"warning: --gpus {args.gpus} with one process")
    torch.cuda.set_device(local)

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
    ms = start.elapsed_time(end) / args.steps
    launches_per_step = 5 + tm.build_kernel_launches + 3  # extent x2, keys, gather, (sort: CUB) ; build ; walk gather/walk/scatter

    # ---- timed: host buffers through the C ABI (end to end) ----
    pos_h = torch.from_numpy(ic["pos"]).pin_memory()
    mass_h = torch.from_numpy(ic["mass"]).pin_memory()
    st_h = torch.from_numpy(ic["softtype"]).pin_memory()
    old_h = oldacc_d.cpu().pin_memory()
    acc_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    pot_h = torch.empty(n, dtype=torch.float64).pin_memory()
    ni_h = torch.empty(n, dtype=torch.int32).pin_memory()
    compute(L.ptr(old_h), L.MEM_HOST, pos_h, mass_h, st_h, acc_h, pot_h, ni_h)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        compute(L.ptr(old_h), L.MEM_HOST, pos_h, mass_h, st_h, acc_h, pot_h, ni_h)
    end.record(stream)
    torch.cuda.synchronize()
    ms_e2e = start.elapsed_time(end) / args.steps

    # ---- PM long-range force of the same particles (PMGRID = 512), device-resident ----
    pm_acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    pm_ms = []
    for k in range(4):
        s = lib.gpugrav_pm_periodic(ctx, 512, n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(pm_acc), None, L.MEM_DEVICE)
        if s != 0:
            raise L.GpuGravError(s, lib.gpugrav_last_error(ctx).decode())
        if k > 0:
            pm_ms.append(tree.timings().pm_ms)
    pm = {"pmgrid": 512, "ms": float(np.mean(pm_ms)), "mesh": "FP64, cuFFT D2Z/Z2D",
          "treepm_ms_per_step": ms + float(np.mean(pm_ms)),
          "note": "tree short-range step (ms_per_step) + PM long-range force: one full TreePM force computation"}
    del pm_acc

    # ---- accuracy against FP64 direct summation on 8192 sampled targets ----
    rng = np.random.default_rng(2004)
    tg = np.sort(rng.choice(n, 8192, replace=False))
    acc_tree = acc_h.numpy()[tg]

    def err_stats(acc_dir):
        return err_stats_of(acc_tree, acc_dir)

    def err_stats_of(acc_tree, acc_dir):
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
    # total force (tree short range + PM long range, PMGRID 512) against the Ewald-corrected direct sum of
    # every pair on 1024 of the targets (FORCETEST's ftrue, gpugrav_direct_split)
    tg_tot = tg[:: max(1, len(tg) // 1024)][:1024]
    pm_acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    s = lib.gpugrav_pm_periodic(ctx, 512, n, L.ptr(pos_d), L.ptr(mass_d), L.ptr(pm_acc), None, L.MEM_DEVICE)
    if s != 0:
        raise L.GpuGravError(s, lib.gpugrav_last_error(ctx).decode())
    a_true, _, a_short, _ = tree.direct_split(tg_tot)
    a_treepm = acc_h.numpy()[tg_tot] + pm_acc.cpu().numpy()[tg_tot]
    del pm_acc
    acc_stats["total_force"] = dict(err_stats_of(a_treepm, a_true), targets=int(len(tg_tot)),
                                    reference="tree (FP32 walk) + PM (PMGRID 512) against the Ewald-corrected FP64 direct "
                                              "sum of every pair (FORCETEST's ftrue)",
                                    pm_vs_direct_long_range=err_stats_of(a_treepm - acc_h.numpy()[tg_tot], a_true - a_short))

    # ---- precision ablation on the same particles and tree code: the FP32 walk's algorithm with FP64
    # arithmetic, and the per-target FP64 walk (the reference's decisions) at matched accuracy ----
    ablation = None
    if prec == L.PREC_FP32 and not args.no_ablation:
        ablation = {}
        for name, p_mode, alpha, steps in (("fp64_group_walk", L.PREC_FP64_GROUP, args.err_tol_force_acc, 3),
                                           ("fp64_per_target_walk", L.PREC_FP64, ABLATION_FP64_ALPHA, 2)):
            pa = ics.params_for(ic, precision=p_mode, err_tol_theta=0.0, err_tol_force_acc=alpha)
            tree.set_params(pa)
            compute(L.ptr(oldacc_d), L.MEM_DEVICE, pos_d, mass_d, st_d, acc_d, pot_d, ni_d)  # warm-up
            torch.cuda.synchronize()
            start.record(stream)
            wl = []
            for _ in range(steps):
                compute(L.ptr(oldacc_d), L.MEM_DEVICE, pos_d, mass_d, st_d, acc_d, pot_d, ni_d)
                wl.append(tree.timings().walk_ms)
            end.record(stream)
            torch.cuda.synchronize()
            ms_a = start.elapsed_time(end) / steps
            ia_a = tree.timings().interactions
            acc_a = acc_d.cpu().numpy()[tg]
            ablation[name] = {"err_tol_force_acc": alpha, "steps": steps, "ms_per_step": ms_a,
                              "value": n / (ms_a * 1e-3), "walk_ms": float(np.mean(wl)), "interactions_per_particle": ia_a / n,
                              "accuracy": {k: v for k, v in err_stats_of(acc_a, acc_cut).items() if k in ("rms_rel", "p99_rel")}}
        v32 = n / (ms * 1e-3)
        ablation["fp32_over_fp64_group"] = v32 / ablation["fp64_group_walk"]["value"]
        ablation["fp32_over_fp64_per_target"] = v32 / ablation["fp64_per_target_walk"]["value"]
        ablation["note"] = ("same particles, device-resident inputs, full step (keys, sort, build, walk); fp64_group_walk: "
                            "the FP32 walk's groups, opening decisions and interaction lists with FP64 arithmetic, at "
                            "the same ErrTolForceAcc; fp64_per_target_walk: the per-target FP64 walk (the reference's "
                            "decisions, bit-exact with it) at the ErrTolForceAcc that brings its RMS error to the FP32 "
                            "walk's")
        prm.precision = prec
        tree.set_params(prm)

    # ---- roofline of the walk kernel (device time measured with CUDA events on its stream) ----
    pk = L.C.c_double(0.0)
    lib.gpugrav_measure_fma_peak(local, prec, L.C.byref(pk))
    peak = float(pk.value)
    walk_s = float(np.mean(walk_ms)) * 1e-3
    ia = float(np.mean(inter))
    achieved = FLOPS_PER_INTERACTION * ia / walk_s / 1e12
    roofline = {"bound": "fp32" if prec == L.PREC_FP32 else "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None,
                "traffic": WALK32_DRAM_BYTES_PER_PARTICLE * n if prec == L.PREC_FP32 else None,
                "traffic_source": "ncu capture of the N=2^21 zoom box walk scaled by particle count",
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
        "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if prec == L.PREC_FP32 else "f64", "data": "synthetic (seeded zoom box, arepo_b200/ics.py)",
        "config": workload_config(lh, args.precision, args.err_tol_force_acc),
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": ms_e2e, "h2d_bytes_per_step": n * (24 + 8 + 1 + 4),
                "d2h_bytes_per_step": n * (24 + 8 + 4)},
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clk.report(),
        "accuracy": acc_stats,
        "interactions_per_particle": ia / n,
        "pm": pm,
        "precision_ablation": ablation,
        "tree": {"num_nodes": int(info.num_nodes), "max_depth": int(info.max_depth),
                 "topnodes": int(info.num_topnodes)},
    }
    if not args.no_cpu_baseline:
        try:
            model, ncpu = cpu_info()
            d = run_cpu_reference(max(1, ncpu or 1), args.err_tol_force_acc, 2, log2_half=lh)
            v, step = cpu_reference_value(d, d["walk_s"][-1])
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": d["procs"], "kind": "reference",
                                    "sample": cpu_sample_text(d, model),
                                    "detail": dict(d, full_step_s_extrapolated=step)}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    tree.close()
    del pos_d, mass_d, st_d, acc_d, pot_d, ni_d, oldacc_d
    torch.cuda.empty_cache()
    if not args.no_serving:
        line["serving"] = serving_leg(args, local)
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--err-tol-force-acc", type=float, default=6e-5,
                    help="ErrTolForceAcc of the timed relative-criterion steps; 6e-5 keeps the FP32 walk's RMS force "
                         "error below 1e-3 on the zoom box (the metric's accuracy bar: 9.4e-4)")
    ap.add_argument("--log2-half", type=int, default=23, help="log2 of each species' count (23 -> N=2^24)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-ablation", action="store_true", help="skip the FP64 forms of the walk")
    ap.add_argument("--sharded", action="store_true",
                    help="use the sharded multi-GPU form also with one rank (it is the default for N > 1)")
    ap.add_argument("--serve-requests", type=int, default=160, help="requests in the Poisson serving stream")
    ap.add_argument("--serve-compare", type=int, default=48,
                    help="first requests of the stream timed batched and one at a time")
    ap.add_argument("--serve-load", type=float, default=0.7,
                    help="Poisson arrival rate as a fraction of the batched all-at-once request rate")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 or args.sharded:
        return sharded_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
