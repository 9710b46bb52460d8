#!/usr/bin/env python
"""Benchmark of the SRC/MPCD time step on B200: particle-steps/s of the FP64 plain form.

Workload: the large plain-FP64 Poiseuille channel, 2048 x 512 cells (a = 0.2), 10 particles
per cell (10,485,760 particles), dt = 0.1, alpha = 130 deg, body force 1e-3 along +x,
periodic x, thermalising walls at y = 0 and y = Ly, 10 x 10 redistribution tiles with a
shifted second pass, closure stiffness 1. Synthetic seeded state (uniform positions,
Maxwellian velocities with kT = 1, mean removed). The state (378 MB) is larger than L2
(126 MB), so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours: W warm-up steps, then K steps timed with CUDA events on the context's stream,
bracketed by a barrier and a device synchronisation on every rank; value = all ranks'
particle-steps / max-over-ranks time. Under torchrun every rank advances its own replica on
its own GPU (the step has no cross-replica exchange).

reference: the unmodified reference (oracle/_ref/ref_sampled, built from the reference's
own sources) on the host cores, on a bounded sample of the same workload: one full step of
everything but the zone passes, plus a sample of zones per pass scaled to all zones.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200: FP64 plain vs FP32+learned closure, at ≤1% profile err"
UNIT = "particle-steps/s"
WORKLOADS = {
    # the benchmark workload: the large plain-FP64 channel
    "channel_2048x512_ppc10": dict(name="channel_2048x512_ppc10", Nx=2048, Ny=512, ppc=10),
    # a smaller channel of the same physics, for profiler captures (state 47 MB)
    "channel_512x256_ppc10": dict(name="channel_512x256_ppc10", Nx=512, Ny=256, ppc=10),
    # the precision-form domain at full size, here in the plain FP64 form (83.9 M particles)
    "channel_4096x1024_ppc20": dict(name="channel_4096x1024_ppc20", Nx=4096, Ny=1024, ppc=20),
    # the reference's own benchmark case (50x50 cells, 25,000 particles)
    "channel_50x50_ppc10": dict(name="channel_50x50_ppc10", Nx=50, Ny=50, ppc=10),
    # batched ensemble: 256 independent channels, Nx ~ U[32,512], Ny ~ U[16,128],
    # ppc ~ U[5,20], bodyForceX log-uniform in [1e-4, 1e-2], one initial-state seed each
    "ensemble_256": dict(name="ensemble_256", replicas=256, seed=2024),
}
WORKLOAD = WORKLOADS["channel_2048x512_ppc10"]
DATA = "synthetic: seeded uniform positions, Maxwellian velocities (kT=1, mean removed)"
# algorithmic bytes per particle (P) and per cell (C) of one launch of each phase's main
# kernel, FP64 plain form: the least each launch must read and write
PHASE_BYTES = {
    "stream_bc": (72, 0),       # read x,v 32 B; write x,v 32 B; write 2 cell ids 8 B
    "zone_pass": (68, 8),       # read slot 4, x 16, v 16; write x 16, v 16 | counts 8 per cell
    "kick_resort": (76, 32),    # read slot 4, x,v 32, pid 4; write x,v,pid 36 | duR, duEOS 32 per cell
    "collide": (36, 16),        # read slot 4, v 16; write v 16 | segment starts 16 per cell
    "cell_index": (40, 24),     # cid, pos 8; cid, pos, pid 12 + key 8; key 8 + slot 4 | count, scan 24
    "ref_fields": (20, 96),     # read slot 4, v 16 | 10 field arrays + start
    "closure_cells": (20, 64),
}
# the same for the FP32 precision form: 20 B of state per particle (cell 4, FP32 offset 8,
# FP32 velocity 8) instead of 32
PHASE_BYTES_F32 = {
    "stream_bc": (48, 0),       # read cell, offset, v 20 B; write 20 B; write 2 cell ids 8 B
    "zone_pass": (44, 8),       # read slot 4, state 20; write state 20 | counts 8 per cell
    "kick_resort": (52, 32),    # read slot 4, state 20, pid 4; write state, pid 24 | 32 per cell
    "collide": (20, 16),        # read slot 4, v 8; write v 8 | segment starts 16 per cell
    "cell_index": (40, 24),     # as the FP64 form: ids, positions in cells, keys and slots
    "ref_fields": (12, 96),     # read slot 4, v 8 | 10 field arrays + start
    "closure_cells": (12, 64),
}
LAUNCHES_PER_STEP = {"zone_pass": 2, "cell_index": 4}


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self):
        return time.time()

    def stop(self, t0, t1):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l for (t, l) in self.lines if t0 - 0.15 <= t <= t1 + 0.15] or [l for (_, l) in self.lines[-3:]]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            f = [x.strip() for x in r.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for k, val in zip(names, f[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus):
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return world, rank, local, dist, torch
    return 1, 0, 0, None, None


def barrier(dist, torch):
    if dist is not None:
        dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()


def reduce_max(x, dist, torch):
    """Max over ranks (every rank times its own replica; the job takes the slowest)."""
    if dist is None:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, n_per_rank, steps, t_max):
    """particle-steps/s of the whole job: every rank advances its own n-particle replica."""
    return world * n_per_rank * steps / t_max


def config_dict(p, world, closure="plain", form="f64"):
    state_bytes = 36 if form == "f64" else 24
    return {
        "workload": WORKLOAD["name"], "Nx": p["Nx"], "Ny": p["Ny"], "particles_per_cell": WORKLOAD["ppc"],
        "n_particles": p["n"], "n_cells": p["Nc"],
        "form": ("plain_" if closure == "plain" else "learned_closure_") + form,
        "state": "FP64 x, v" if form == "f64" else "int32 cell, FP32 offset in cell, FP32 v (FP64 arithmetic)",
        "dt": p["dt"],
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "l2_policy": f"state ({state_bytes * p['n'] / 1e6:.0f} MB) vs L2 126 MB; no flush",
    }


def cpu_baseline_port(p, x, v):
    """The oracle port (single thread) on one full step of the workload."""
    from tests.oracle_libs import Oracle
    O = Oracle()
    t0 = time.perf_counter()
    O.step(p, x, v, 1)
    dt = time.perf_counter() - t0
    return {"value": p["n"] / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one full step of {WORKLOAD['name']} ({p['n']} particles) with the C oracle, one thread: {dt:.1f} s"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_traffic(kernel, form="f64"):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)
        e = d.get(kernel)
        if e and e.get("workload") == WORKLOAD["name"] and e.get("form", "f64") == form:
            return float(e["bytes_per_launch"])
    except (OSError, ValueError):
        pass
    return None


def run_ours(args):
    from src_incompressible_openmp_b200 import native
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

    world, rank, local, dist, torch = dist_setup(args.gpus)
    p = poiseuille_params(WORKLOAD["Nx"], WORKLOAD["Ny"], WORKLOAD["ppc"])
    x, v = uniform_state(p, 1 + rank)
    learned = None
    if args.closure == "learned":
        learned = learned_network(args, local)
    ctx = native.Context(p, device=local, form=args.form)
    ctx.set_state(x, v)
    W, K = args.warmup, args.steps
    if learned is not None:
        # fallback limit: 1.2 x the plain closure's occupancy spread, taken from a plain step
        occ_plain = ctx.step(0, 1, metrics=True)["occStd"]
        ctx.learned_set(learned["params"], 1.2 * occ_plain)
        learned["occ_limit"] = 1.2 * occ_plain
        ctx.step(1, W - 1)
    else:
        ctx.step(0, W)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    l0 = ctx.launch_count()
    barrier(dist, torch)
    t_wall0 = time.time()
    t_dev = ctx.step_timed(W, K)
    barrier(dist, torch)
    t_wall1 = time.time()
    l1 = ctx.launch_count()
    clocks = sampler.stop(t_wall0, t_wall1)
    t_max = reduce_max(t_dev, dist, torch)
    value = whole_job_value(world, p["n"], K, t_max)
    # live per-phase timing (separate run: one synchronisation per step)
    KP = max(1, min(K, args.profile_steps))
    phases = ctx.step_profile(W + K, KP)
    # end-to-end through the C-ABI with pinned host buffers (mpcd_run_jobs): every step is a
    # job that uploads its input state, runs one step and downloads the resulting state; the
    # copies of neighbouring jobs overlap each job's step
    KE = max(1, min(K, args.e2e_steps))
    host = [native.PinnedArray(2 * p["n"]) for _ in range(6)]
    hx, hv = host[0].array, host[1].array
    hx[:] = x
    hv[:] = v
    outs_x = [host[2].array, host[3].array]
    outs_v = [host[4].array, host[5].array]
    # untimed warm-up call: allocates the job staging buffers and copy streams
    ctx.run_jobs([hx] * 2, [hv] * 2, W + K + KP, 1, outs_x, outs_v)
    barrier(dist, torch)
    t0 = time.perf_counter()
    ctx.run_jobs([hx] * KE, [hv] * KE, W + K + KP + 2, 1, [outs_x[k % 2] for k in range(KE)],
                 [outs_v[k % 2] for k in range(KE)])
    barrier(dist, torch)
    te = reduce_max(time.perf_counter() - t0, dist, torch)
    for h in host:
        h.close()
    ctx_stats = ctx.learned_stats()
    e2e = {"value": whole_job_value(world, p["n"], KE, te), "unit": UNIT, "h2d_bytes_per_step": 32 * p["n"],
           "d2h_bytes_per_step": 32 * p["n"], "steps": KE,
           "note": "per step: upload of the input state from pinned host memory, one step, download of the "
                   "resulting state (mpcd_run_jobs: copies of neighbouring steps overlap the step)"}
    ctx.close()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    # roofline of the dominant kernel
    peak, peak_src = measured_peaks()
    table = PHASE_BYTES if args.form == "f64" else PHASE_BYTES_F32
    dom = max((k for k in phases if k in table), key=lambda k: phases[k])
    per_launch_s = phases[dom] / (KP * LAUNCHES_PER_STEP.get(dom, 1))
    bp, bc = table[dom]
    alg = bp * p["n"] + bc * p["Nc"]
    achieved = alg / per_launch_s / 1e9
    bp_step = 256 if args.form == "f64" else 160  # 4 state sweeps, read + write
    step_bytes = bp_step * p["n"] + 128 * p["Nc"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.form, "data": DATA, "config": config_dict(p, world, args.closure, args.form),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": measured_traffic(dom, args.form),
                     "peak_source": peak_src, "algorithmic_bytes_per_launch": alg,
                     "avg_launch_ms": 1e3 * per_launch_s},
        "step_hbm": {"algorithmic_bytes_per_step": step_bytes,
                     "achieved_GBps": step_bytes * K / t_max / 1e9 * world,
                     "note": f"{bp_step} B per particle + 128 B per cell per step"},
        "phases_ms_per_step": {k: 1e3 * t / KP for k, t in phases.items()},
        "e2e": e2e,
        "gpu_launches": int((l1 - l0) * world),
        "clocks": clocks,
    }
    if learned is not None:
        plain_steps, learned_steps, _ = ctx_stats
        line["learned_closure"] = {k: learned[k] for k in learned if k != "params"}
        line["learned_closure"].update({"steps_plain": plain_steps, "steps_learned": learned_steps})
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(p, x, v)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def learned_network(args, device):
    """The learned closure's network: loaded from --network, or collected and trained here on
    the ensemble family (the plain closure's kicks in 200 seeded channels, up to 2 M cells, with
    their mirror images; Adam on the GPU)."""
    import numpy as np

    from src_incompressible_openmp_b200 import learned as L

    if args.network:
        return {"params": np.load(args.network), "source": args.network}
    t0 = time.perf_counter()
    X, Y = L.collect(runs=200, seed=7, warmup=60, steps=20, stride=4, capacity=2_000_000, device=device)
    t1 = time.perf_counter()
    net, losses = L.train(X, Y, epochs=6, device=device)
    t2 = time.perf_counter()
    return {"params": net, "source": "trained in this run", "train_samples": int(len(X)),
            "collect_s": t1 - t0, "train_s": t2 - t1, "final_loss": float(losses[-1])}


def ensemble_params(W):
    """Parameters and initial state seeds of the batched ensemble."""
    from src_incompressible_openmp_b200.cases import ensemble_family

    return ensemble_family(W["replicas"], W["seed"])


def run_ensemble(args):
    """Aggregate particle-steps/s of the batched ensemble (one GPU; rank 0 only)."""
    from src_incompressible_openmp_b200 import native
    from src_incompressible_openmp_b200.cases import uniform_state

    if env_int("RANK", 0) != 0:
        return
    reps = ensemble_params(WORKLOAD)
    B = native.Batch([p for p, _ in reps])
    for i, (p, seed) in enumerate(reps):
        x, v = uniform_state(p, seed)
        B.member(i).set_state(x, v)
    W, K = args.warmup, args.steps
    B.step(0, W)
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = sum(B.member(i).launch_count() for i in range(len(reps)))
    t_wall0 = time.time()
    t_dev = B.step(W, K)
    t_wall1 = time.time()
    l1 = sum(B.member(i).launch_count() for i in range(len(reps)))
    clocks = sampler.stop(t_wall0, t_wall1)
    n_tot = sum(p["n"] for p, _ in reps)
    nc_tot = sum(p["Nc"] for p, _ in reps)
    B.close()
    line = {
        "metric": METRIC, "value": n_tot * K / t_dev, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * t_dev / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: per replica seeded uniform positions, Maxwellian velocities",
        "config": {"workload": WORKLOAD["name"], "replicas": len(reps), "n_particles": n_tot, "n_cells": nc_tot,
                   "form": "plain_f64, one context and stream per replica, steps replayed from CUDA graphs",
                   "parallelism": "single GPU"},
        "step_hbm": {"algorithmic_bytes_per_step": 256 * n_tot + 128 * nc_tot,
                     "achieved_GBps": (256 * n_tot + 128 * nc_tot) * K / t_dev / 1e9},
        "e2e": None, "gpu_launches": int(l1 - l0), "clocks": clocks,
    }
    print(json.dumps(line))


def run_reference(args):
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state, write_case

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    p = poiseuille_params(WORKLOAD["Nx"], WORKLOAD["Ny"], WORKLOAD["ppc"])
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_sampled")
    threads = os.cpu_count() or 1
    x, v = uniform_state(p, 1)
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_sampled was not built (reference sources absent at build time)"}))
        return
    budget = args.reference_budget_s
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as d:
        write_case(d, p, x, v, {"benchmark_nSteps": 1, "benchmark_metricsEvery": 1, "benchmark_dumpSteps": ""})
        runs = []
        t_start = time.time()
        n_warm = min(args.warmup, 1)
        k = 0
        while True:
            r = subprocess.run([exe, os.path.join(d, "params.kv"), os.path.join(d, "in_x.bin"), os.path.join(d, "in_v.bin"),
                                str(threads), "1", str(k + 1)], capture_output=True, text=True)
            if r.returncode != 0:
                print(json.dumps({"impl": "reference", "unavailable": "reference harness failed: " + r.stderr.strip()[-200:]}))
                return
            runs.append(json.loads(r.stdout))
            k += 1
            elapsed = time.time() - t_start
            timed = len(runs) - n_warm
            per = elapsed / len(runs)
            if timed >= args.steps or (timed >= 1 and elapsed + per > budget):
                break
    timed_runs = runs[n_warm:]
    t_step = statistics.mean(r["t_step_extrapolated"] for r in timed_runs)
    value = p["n"] / t_step
    sample = (f"{len(timed_runs)} sampled steps of {WORKLOAD['name']} on {threads} threads: full stream/BC/SRD and closure, "
              f"{timed_runs[0]['base_sampled']}/{timed_runs[0]['base_zones']} base and {timed_runs[0]['shifted_sampled']}/"
              f"{timed_runs[0]['shifted_zones']} shifted zones per step through the reference's own per-zone body, "
              f"scaled to all zones")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": len(timed_runs), "warmup": n_warm, "ms_per_step": 1e3 * t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA, "config": config_dict(p, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phases_s": {k: statistics.mean(r[k] for r in timed_runs) for k in ("t_refbuild", "base_extrapolated", "shifted_extrapolated", "t_closure")},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="channel_2048x512_ppc10")
    ap.add_argument("--closure", choices=["plain", "learned"], default="plain",
                    help="learned: the stencil-MLP closure with the plain closure as fallback")
    ap.add_argument("--network", default=None, help="learned closure parameters (.npy); default: train here")
    ap.add_argument("--form", choices=["f64", "f32"], default="f64",
                    help="f32: the FP32 precision form (FP32 cell-relative positions and velocities)")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.workload]
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif "replicas" in WORKLOAD:
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
