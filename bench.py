#!/usr/bin/env python
"""Benchmark of the SRC/MPCD time step on B200: FP64 plain vs FP32 fast form with the learned
closure, in particle-steps/s, with the fast form's profile error against the plain form.

Workload (default): the Poiseuille channel of 4096 x 1024 cells (a = 0.2) at 20 particles per
cell (83,886,080 particles), dt = 0.1, alpha = 130 deg, body force 1e-3 along +x, periodic x,
thermalising walls at y = 0 and y = Ly, 10 x 10 redistribution tiles with a shifted second
pass, closure stiffness 1. Synthetic seeded state (uniform positions, Maxwellian velocities
with kT = 1, mean removed). The state (3 GB in the plain form) is larger than L2 (126 MB), so
no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

ours: W warm-up steps, then K steps timed with CUDA events on the context's stream,
bracketed by a barrier and a device synchronisation on every rank; value = all ranks'
particle-steps / max-over-ranks time of the FP64 plain form. In the same line, "chosen_form"
gives the same measurement of the fast form (FP32 bins, parallel redistribution) with the
learned closure, its ratio to the plain form, and the L2 error of its time-averaged velocity
profile against the plain form's over --profile-steps steps (averaged over the second half),
beside the plain form's own seed-to-seed difference (the noise floor). Under torchrun every
rank advances its own replica on its own GPU (the step has no cross-replica exchange).

reference: the unmodified reference (built from the reference's own sources by
oracle/Makefile) on the host cores: on the workload, one step of everything but the zone
passes plus a sample of zones per pass scaled to all zones (labelled extrapolated); and, in the
same line, the reference's own benchmark driver on its own 50 x 50 case for all 1,500 steps,
timed in full.
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
    # the benchmark workload: the target's channel (83.9 M particles)
    "channel_4096x1024_ppc20": dict(name="channel_4096x1024_ppc20", Nx=4096, Ny=1024, ppc=20),
    # the large plain-FP64 channel (10.5 M particles)
    "channel_2048x512_ppc10": dict(name="channel_2048x512_ppc10", Nx=2048, Ny=512, ppc=10),
    # a smaller channel of the same physics, for profiler captures (state 47 MB)
    "channel_512x256_ppc10": dict(name="channel_512x256_ppc10", Nx=512, Ny=256, ppc=10),
    # the reference's own benchmark case (50x50 cells, 25,000 particles)
    "channel_50x50_ppc10": dict(name="channel_50x50_ppc10", Nx=50, Ny=50, ppc=10),
    # batched ensemble: 256 independent channels, Nx ~ U[32,512], Ny ~ U[16,128],
    # ppc ~ U[5,20], bodyForceX log-uniform in [1e-4, 1e-2], one initial-state seed each
    "ensemble_256": dict(name="ensemble_256", replicas=256, seed=2024),
}
WORKLOAD = WORKLOADS["channel_4096x1024_ppc20"]
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
# the fast form: FP32 bins (offset 8, velocity 8, id 4 bytes per particle); bytes per step of
# each phase (its kernels together)
PHASE_BYTES_FAST = {
    "stream_bc": (40, 16),      # read 20 B, write 20 B | count read, count claimed, kick 16 per cell
    "collide": (28, 4),         # tiles read offset, velocity, id 20; write velocity 8 | count
    "zone_pass": (20, 128),     # both passes: base reads velocity and id 12, rewrites velocities 8 |
                                # counts, summaries, momentum sums and reference sums 128 per cell
    "closure_cells": (0, 92),   # reference and red sums 48 + counts 4; pdrive, duRepair, beta terms 40
    "kick_resort": (0, 48),     # pressure drive and duRepair read 24 (+ stencil), kick written 8
}
LAUNCHES_PER_STEP = {"zone_pass": 2, "cell_index": 4}
LAUNCHES_PER_STEP_FAST = {}


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


def config_dict(p, world, form="plain_f64"):
    return {
        "workload": WORKLOAD["name"], "Nx": p["Nx"], "Ny": p["Ny"], "particles_per_cell": WORKLOAD["ppc"],
        "n_particles": p["n"], "n_cells": p["Nc"], "form": form, "state": "FP64 x, v", "dt": p["dt"],
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "l2_policy": f"state ({36 * p['n'] / 1e6:.0f} MB) vs L2 126 MB; no flush",
        "metricsEvery": "none inside the timed steps (one metrics row after them)",
    }


def cpu_baseline_port(p):
    """The oracle port (single thread) on one full step of a bounded sub-case of the workload
    (the same channel physics and density on a quarter of the cells in each direction when the
    workload is large); the rate per particle does not depend on the domain size."""
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state
    from tests.oracle_libs import Oracle
    sub = p
    if p["n"] > 12_000_000:
        sub = poiseuille_params(p["Nx"] // 4, p["Ny"] // 2, WORKLOAD["ppc"])
    x, v = uniform_state(sub, 1)
    O = Oracle()
    t0 = time.perf_counter()
    O.step(sub, x, v, 1)
    dt = time.perf_counter() - t0
    return {"value": sub["n"] / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one full step of the {sub['Nx']}x{sub['Ny']} channel at {WORKLOAD['ppc']} per cell "
                      f"({sub['n']} particles) with the C oracle, one thread: {dt:.1f} s"}


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
        e = d.get(kernel if form == "f64" else f"{kernel}:{form}")
        if e and e.get("workload") == WORKLOAD["name"] and e.get("form", "f64") == form:
            return float(e["bytes_per_launch"])
    except (OSError, ValueError):
        pass
    return None


def roofline(phases, KP, p, table, form):
    """Roofline of the dominant kernel: its algorithmic bytes per launch over its live launch time."""
    peak, peak_src = measured_peaks()
    dom = max((k for k in phases if k in table), key=lambda k: phases[k])
    launches = (LAUNCHES_PER_STEP if form == "f64" else LAUNCHES_PER_STEP_FAST).get(dom, 1)
    per_launch_s = phases[dom] / (KP * launches)
    bp, bc = table[dom]
    alg = bp * p["n"] + bc * p["Nc"]
    achieved = alg / per_launch_s / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": measured_traffic(dom, form), "peak_source": peak_src, "algorithmic_bytes_per_launch": alg,
            "avg_launch_ms": 1e3 * per_launch_s}


def timed_steps(native, ctx, W, K, KP, dist, torch, world, n, local):
    """W warm-up steps, K timed steps (device time, max over ranks), KP profiled steps."""
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
    phases = ctx.step_profile(W + K, KP)
    return t_max, clocks, l1 - l0, phases


def profile_run(native, p, seed, form, steps, network=None, occ_limit=0.0, device=0):
    """Velocity profile across the channel, averaged over the second half of `steps` steps."""
    from src_incompressible_openmp_b200.cases import uniform_state
    x, v = uniform_state(p, seed)
    with native.Context(p, device=device, form=form) as ctx:
        ctx.set_state(x, v)
        if network is not None:
            ctx.learned_set(network, occ_limit)
        ctx.step(0, steps // 2)
        ctx.profile_reset(True)
        m = ctx.step(steps // 2, steps - steps // 2, metrics=True)
        ux, k = ctx.profile_read()
        stats = ctx.learned_stats() if network is not None else None
    return ux, m, stats


def run_ours(args):
    import numpy as np

    from src_incompressible_openmp_b200 import native
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

    world, rank, local, dist, torch = dist_setup(args.gpus)
    p = poiseuille_params(WORKLOAD["Nx"], WORKLOAD["Ny"], WORKLOAD["ppc"])
    x, v = uniform_state(p, 1 + rank)
    W, K = args.warmup, args.steps
    KP = max(1, min(K, args.profile_steps))
    # ---- the FP64 plain form (value)
    ctx = native.Context(p, device=local, form="f64")
    ctx.set_state(x, v)
    t_max, clocks, launches, phases = timed_steps(native, ctx, W, K, KP, dist, torch, world, p["n"], local)
    value = whole_job_value(world, p["n"], K, t_max)
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
    ctx.run_jobs([hx] * 2, [hv] * 2, W + K + KP, 1, outs_x, outs_v)  # untimed: allocates the staging
    barrier(dist, torch)
    t0 = time.perf_counter()
    ctx.run_jobs([hx] * KE, [hv] * KE, W + K + KP + 2, 1, [outs_x[k % 2] for k in range(KE)],
                 [outs_v[k % 2] for k in range(KE)])
    barrier(dist, torch)
    te = reduce_max(time.perf_counter() - t0, dist, torch)
    for h in host:
        h.close()
    ctx.close()
    e2e = {"value": whole_job_value(world, p["n"], KE, te), "unit": UNIT, "h2d_bytes_per_step": 32 * p["n"],
           "d2h_bytes_per_step": 32 * p["n"], "steps": KE,
           "note": "per step: upload of the input state from pinned host memory, one step, download of the "
                   "resulting state (mpcd_run_jobs: copies of neighbouring steps overlap the step); bound by the "
                   "host link at 32 B per particle each way"}
    # ---- the chosen form: fast form with the learned closure
    chosen = None
    if args.chosen != "none":
        net = learned_network(args, local) if args.chosen == "learned" else None
        cf = native.Context(p, device=local, form="fast")
        cf.set_state(x, v)
        occ_limit = 0.0
        if net is not None:
            occ_plain = cf.step(0, 1, metrics=True)["occStd"]
            occ_limit = 1.2 * occ_plain
            cf.learned_set(net["params"], occ_limit)
        tf, clocks_f, launches_f, phases_f = timed_steps(native, cf, W, K, KP, dist, torch, world, p["n"], local)
        stats = cf.learned_stats() if net is not None else None
        cf.close()
        vf = whole_job_value(world, p["n"], K, tf)
        chosen = {
            "form": "fast_f32_" + args.chosen + "_closure", "value": vf, "unit": UNIT, "ms_per_step": 1e3 * tf / K,
            "ratio_vs_plain": vf / value,
            "state": "per-cell bins: FP32 offset in cell, FP32 velocity on the 2^-20 grid, particle id (int64 cell sums)",
            "phases_ms_per_step": {k: 1e3 * t / KP for k, t in phases_f.items() if t > 0},
            "roofline": roofline({k: t for k, t in phases_f.items() if t > 0}, KP, p, PHASE_BYTES_FAST, "fast"),
            "step_hbm": {"algorithmic_bytes_per_step": 128 * p["n"] + 128 * p["Nc"],
                         "achieved_GBps": (128 * p["n"] + 128 * p["Nc"]) * K / tf / 1e9 * world,
                         "note": "128 B per particle + 128 B per cell per step (FP32 state)"},
            "gpu_launches": int(launches_f * world), "clocks": clocks_f,
        }
        if net is not None:
            chosen["learned_closure"] = {k: v for k, v in net.items() if k != "params"}
            chosen["learned_closure"].update({"occ_limit": occ_limit, "steps_plain": stats[0], "steps_learned": stats[1]})
        if args.profile_steps_long > 0 and world == 1:
            S = args.profile_steps_long
            pa, ma, _ = profile_run(native, p, 1, "f64", S, device=local)
            pb, mb, _ = profile_run(native, p, 2, "f64", S, device=local)
            pc, mc, st2 = profile_run(native, p, 1, "fast", S, None if net is None else net["params"], occ_limit, local)
            na = float(np.linalg.norm(pa))
            chosen["profile"] = {
                "steps": S, "averaged_over": f"steps {S // 2 + 1}-{S}",
                "profile_l2_err": float(np.linalg.norm(pc - pa)) / na,
                "noise_floor": float(np.linalg.norm(pb - pa)) / na,
                "noise_floor_note": "plain form, initial state seed 2 against seed 1",
                "mean_ux_plain": float(np.mean(pa)), "mean_ux_chosen": float(np.mean(pc)),
                "meanKinetic_plain": ma["meanKinetic"], "meanKinetic_chosen": mc["meanKinetic"],
                "occStd_plain": ma["occStd"], "occStd_chosen": mc["occStd"],
            }
            if st2 is not None:
                chosen["profile"]["steps_learned"] = st2[1]
                chosen["profile"]["steps_plain_fallback"] = st2[0]
            if net is not None:
                # what the network replaces: the same run with a zero network (no EOS kick in
                # the bulk; the walls keep the plain one, the repair kick stays)
                from src_incompressible_openmp_b200 import learned as L
                pz, mz, _ = profile_run(native, p, 1, "fast", S, L.zero_network(), occ_limit, local)
                chosen["profile"]["profile_l2_err_no_eos_kick"] = float(np.linalg.norm(pz - pa)) / na
                chosen["profile"]["occStd_no_eos_kick"] = mz["occStd"]
                chosen["profile"]["meanKinetic_no_eos_kick"] = mz["meanKinetic"]
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    step_bytes = 256 * p["n"] + 128 * p["Nc"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": DATA, "config": config_dict(p, world),
        "roofline": roofline(phases, KP, p, PHASE_BYTES, "f64"),
        "step_hbm": {"algorithmic_bytes_per_step": step_bytes,
                     "achieved_GBps": step_bytes * K / t_max / 1e9 * world,
                     "note": "256 B per particle + 128 B per cell per step"},
        "phases_ms_per_step": {k: 1e3 * t / KP for k, t in phases.items()},
        "e2e": e2e,
        "gpu_launches": int(launches * world),
        "clocks": clocks,
    }
    if chosen is not None:
        line["chosen_form"] = chosen
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(p)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def learned_network(args, device):
    """The fast form's learned closure: loaded from --network, or collected and trained here on
    the ensemble family (the fast form's plain EOS kicks in 200 seeded channels, up to 2 M
    cells, with their mirror images; Adam on the GPU)."""
    import numpy as np

    from src_incompressible_openmp_b200 import learned as L

    if args.network:
        return {"params": np.load(args.network), "source": args.network}
    t0 = time.perf_counter()
    X, Y = L.collect(runs=200, seed=7, warmup=60, steps=20, stride=4, capacity=2_000_000, device=device, form="fast")
    t1 = time.perf_counter()
    net, losses = L.train(X, Y, epochs=6, device=device, form="fast")
    t2 = time.perf_counter()
    held = L.unexplained(net, X[::97], Y[::97])
    return {"params": net, "source": "trained in this run (fast form, ensemble family, 200 channels)",
            "train_samples": int(len(X)), "collect_s": t1 - t0, "train_s": t2 - t1, "final_loss": float(losses[-1]),
            "unexplained_variance_train_sample": held}


def ensemble_params(W):
    """Parameters and initial state seeds of the batched ensemble."""
    from src_incompressible_openmp_b200.cases import ensemble_family

    return ensemble_family(W["replicas"], W["seed"])


def _ensemble_batch(native, reps, form, seed_shift=0):
    """A batch of the ensemble's replicas with their initial states (seed + seed_shift)."""
    from src_incompressible_openmp_b200.cases import uniform_state

    B = native.Batch([p for p, _ in reps], form=form)
    for i, (p, seed) in enumerate(reps):
        x, v = uniform_state(p, seed + seed_shift)
        B.member(i).set_state(x, v)
    return B


def _ensemble_flux(B, reps, step0, rounds, every):
    """Per replica the flux Qx = meanUx * Ly (src/main_benchmark_poiseuille_openmp_profiled_
    shifted_profiled.cpp:124-126: meanUx the mean over cells of the cell mean vx), averaged over
    `rounds` states taken every `every` steps after step0."""
    import numpy as np

    q = np.zeros(len(reps))
    for k in range(rounds):
        B.step(step0 + k * every, every)
        for i, (p, _) in enumerate(reps):
            x, v = B.member(i).get_state()
            ax, ay = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
            ix = np.clip(np.floor(x[0::2] / ax).astype(np.int64), 0, p["Nx"] - 1)
            iy = np.clip(np.floor(x[1::2] / ay).astype(np.int64), 0, p["Ny"] - 1)
            c = iy + p["Ny"] * ix
            n = np.bincount(c, minlength=p["Nc"])
            sx = np.bincount(c, weights=v[0::2], minlength=p["Nc"])
            ux = np.where(n > 0, sx / np.maximum(n, 1), 0.0)
            q[i] += ux.mean() * p["Ly"] / rounds
    return q


def run_ensemble(args):
    """Aggregate particle-steps/s of the batched ensemble (one GPU; rank 0 only): the FP64 plain
    batch as the line's value, the fast-form batch beside it, and each replica's flux error of
    the fast form against FP64."""
    import numpy as np
    from src_incompressible_openmp_b200 import native

    if env_int("RANK", 0) != 0:
        return
    reps = ensemble_params(WORKLOAD)
    W, K = args.warmup, args.steps
    n_tot = sum(p["n"] for p, _ in reps)
    nc_tot = sum(p["Nc"] for p, _ in reps)
    rounds, every = 5, 10
    arms = {}
    for form in ("f64", "fast"):
        B = _ensemble_batch(native, reps, form)
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
        flux = _ensemble_flux(B, reps, W + K, rounds, every)
        B.close()
        arms[form] = dict(t=t_dev, launches=int(l1 - l0), clocks=clocks, flux=flux)
    # the noise floor: the FP64 batch from other initial states, against the first
    B = _ensemble_batch(native, reps, "f64", seed_shift=5000)
    B.step(0, W + K)
    flux_other = _ensemble_flux(B, reps, W + K, rounds, every)
    B.close()
    q64, qf = arms["f64"]["flux"], arms["fast"]["flux"]
    scale = np.maximum(np.abs(q64), 1e-12)
    err = np.abs(qf - q64) / scale
    floor = np.abs(flux_other - q64) / scale
    g = np.array([p["bodyForceX"] for p, _ in reps])
    strong = g >= np.median(g)
    t64, tf = arms["f64"]["t"], arms["fast"]["t"]
    line = {
        "metric": METRIC, "value": n_tot * K / t64, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * t64 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: per replica seeded uniform positions, Maxwellian velocities",
        "config": {"workload": WORKLOAD["name"], "replicas": len(reps), "n_particles": n_tot, "n_cells": nc_tot,
                   "form": "plain_f64, one context and stream per replica, steps replayed from CUDA graphs",
                   "parallelism": "single GPU"},
        "step_hbm": {"algorithmic_bytes_per_step": 256 * n_tot + 128 * nc_tot,
                     "achieved_GBps": (256 * n_tot + 128 * nc_tot) * K / t64 / 1e9},
        "e2e": None, "gpu_launches": arms["f64"]["launches"], "clocks": arms["f64"]["clocks"],
        "fast_batch": {
            "form": "fast form (FP32 state, int64 cell sums), every phase one launch for all replicas",
            "value": n_tot * K / tf, "unit": UNIT, "ms_per_step": 1e3 * tf / K, "ratio_vs_f64_batch": t64 / tf,
            "gpu_launches": arms["fast"]["launches"], "launches_per_step": arms["fast"]["launches"] / K,
            "clocks": arms["fast"]["clocks"],
            "flux_error": {
                "definition": "per replica |Qx_fast - Qx_f64| / |Qx_f64|, Qx = meanUx * Ly averaged over "
                              f"{rounds} states every {every} steps after step {W + K}, both forms from the same "
                              "initial state; noise floor: the FP64 batch from other initial states",
                "median": float(np.median(err)), "p90": float(np.percentile(err, 90)),
                "median_noise_floor": float(np.median(floor)), "p90_noise_floor": float(np.percentile(floor, 90)),
                "median_upper_half_forcing": float(np.median(err[strong])),
                "median_noise_floor_upper_half_forcing": float(np.median(floor[strong])),
                "aggregate_signed": float(np.sum(qf - q64) / np.sum(np.abs(q64))),
                "aggregate_signed_noise_floor": float(np.sum(flux_other - q64) / np.sum(np.abs(q64))),
            },
        },
    }
    print(json.dumps(line))


def reference_measured_leg(threads):
    """The reference's own profiled benchmark driver (oracle/_ref/ref_bench, unmodified) on its
    own case, 50 x 50 cells at 10 per cell (25,000 particles), all 1,500 steps, timed in full."""
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state, write_case
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    if not os.path.exists(exe):
        return None
    p = poiseuille_params(50, 50, 10)
    x, v = uniform_state(p, 1)
    steps = 1500
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as d:
        write_case(d, p, x, v, {"benchmark_nSteps": steps, "benchmark_metricsEvery": 100, "benchmark_dumpSteps": ""})
        c = os.path.join(d, "")
        t0 = time.perf_counter()
        r = subprocess.run([exe, c + "params.kv", c + "in_x.bin", c + "in_v.bin", c + "in_type.bin", c + "in_r0.bin",
                            c + "out", "0", "0", str(threads)], capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"unavailable": "reference driver failed: " + r.stderr.strip()[-200:]}
        kv = {}
        with open(c + "out_runout.kv") as f:
            for line in f:
                if "=" in line:
                    k, val = line.strip().split("=", 1)
                    kv[k] = val
    per_step = float(kv.get("timePerStepMean", wall / steps))
    return {"workload": "channel_50x50_ppc10 (the reference's own case)", "steps": steps, "threads": threads,
            "value": p["n"] / per_step, "unit": UNIT, "s_per_step": per_step, "wall_s": wall,
            "note": "timePerStepMean of the driver's own _runout.kv (step loop only, metrics every 100 steps); "
                    "measured, not extrapolated"}


def run_reference(args):
    from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state, write_case

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    p = poiseuille_params(WORKLOAD["Nx"], WORKLOAD["Ny"], WORKLOAD["ppc"])
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_sampled")
    threads = os.cpu_count() or 1
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_sampled was not built (reference sources absent at build time)"}))
        return
    measured = reference_measured_leg(threads)
    x, v = uniform_state(p, 1)
    budget = args.reference_budget_s
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as d:
        write_case(d, p, x, v, {"benchmark_nSteps": 1, "benchmark_metricsEvery": 1, "benchmark_dumpSteps": ""})
        del x, v
        runs = []
        t_start = time.time()
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
            per = elapsed / len(runs)
            # each sampled step is a one-shot CPU computation: no warm-up; stop at the budget
            if len(runs) >= args.steps or elapsed + per > budget:
                break
    t_step = statistics.mean(r["t_step_extrapolated"] for r in runs)
    value = p["n"] / t_step
    sample = (f"{len(runs)} sampled steps of {WORKLOAD['name']} on {threads} threads: full stream/BC/SRD and closure, "
              f"{runs[0]['base_sampled']}/{runs[0]['base_zones']} base and {runs[0]['shifted_sampled']}/"
              f"{runs[0]['shifted_zones']} shifted zones per step through the reference's own per-zone body, "
              f"scaled to all zones (extrapolated)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": len(runs), "warmup": 0, "ms_per_step": 1e3 * t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA, "config": config_dict(p, 1),
        "extrapolated": True,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phases_s": {k: statistics.mean(r[k] for r in runs) for k in ("t_refbuild", "base_extrapolated", "shifted_extrapolated", "t_closure")},
    }
    if measured is not None:
        line["measured_reference_case"] = measured
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
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="channel_4096x1024_ppc20")
    ap.add_argument("--chosen", choices=["learned", "plain", "none"], default="learned",
                    help="the chosen form's closure (fast form): learned (stencil MLP with the plain "
                         "closure as fallback), plain, or none (skip the chosen form)")
    ap.add_argument("--network", default=None, help="learned closure parameters (.npy); default: train here")
    ap.add_argument("--profile-steps-long", type=int, default=2000,
                    help="steps of the profile-error runs (0: skip); the profile is averaged over the second half")
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
