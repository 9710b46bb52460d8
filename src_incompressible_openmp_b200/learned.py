"""Learned closure workflow: collect (features, target) pairs from the plain closure, train the
stencil MLP on the GPU, and compare it in deployment with the plain closure and with no closure
kick at all.

Everything that computes runs in libmpcd_b200.so through the C-ABI (mpcd_learned_*): sample
collection inside the device step, training with the library's BF16/FP32 forward, backward and
Adam kernels, inference with its tcgen05 kernel. This module only sequences the calls.

    python -m src_incompressible_openmp_b200.learned --runs 200 --out net.npy

trains on the ensemble family (cases.ensemble_family) and writes the parameter array
(MPCD_LEARNED_PARAMS float32 values) that native.Context.learned_set takes.
"""
import argparse
import time

import numpy as np

from . import native
from .cases import ensemble_family, uniform_state


def collect(runs=200, seed=7, warmup=60, steps=20, stride=4, capacity=None, log=None, device=0, form="f64"):
    """Samples from `runs` channels of the ensemble family: each runs `warmup` plain steps, then
    `steps` steps whose closure is sampled at every stride-th cell. Returns (X, Y) float32.
    form "fast": the fast form's closure, whose network sees the collided state's occupancy,
    kinetic pressure and mean vx and predicts the EOS kick."""
    Xs, Ys, total = [], [], 0
    for r, (p, s) in enumerate(ensemble_family(runs, seed)):
        x, v = uniform_state(p, s)
        with native.Context(p, device, form=form) as ctx:
            ctx.set_state(x, v)
            ctx.step(0, warmup)
            X, Y = ctx.learned_samples(warmup, steps, stride)
        Xs.append(X)
        Ys.append(Y)
        total += len(X)
        if log:
            log(f"run {r}: {p['Nx']}x{p['Ny']} ppc {p['n'] // p['Nc']} -> {len(X)} samples ({total} total)")
        if capacity and total >= capacity:
            break
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    if capacity:
        X, Y = X[:capacity], Y[:capacity]
    return X, Y


def _mirror_index():
    """Stencil point permutations of the mirrors x -> -x and y -> -y (point = 5 (dy+2) + dx+2)."""
    k = np.arange(25)
    dy, dx = k // 5, k % 5
    return 5 * dy + (4 - dx), 5 * (4 - dy) + dx


def mirrored(X, Y, form="f64"):
    """The samples with their mirror images in x, in y and in both: the closure commutes with
    the channel's reflections (a reflected cell neighbourhood gets the reflected kick). Feature
    channels 1 and 2 are Ux and Uy (plain and precision forms) or the kinetic pressure and Ux
    (fast form): a reflection negates the velocity channels along its axis."""
    flipx_ch, flipy_ch = ((1,), (2,)) if form != "fast" else ((2,), ())
    mx, my = _mirror_index()
    outX, outY = [X], [Y]
    for flip_x, flip_y in ((True, False), (False, True), (True, True)):
        perm = np.arange(25)
        if flip_x:
            perm = perm[mx]
        if flip_y:
            perm = perm[my]
        Z = np.concatenate([X[:, perm], X[:, 25 + perm], X[:, 50 + perm]], axis=1)
        W = Y.copy()
        if flip_x:
            for ch in flipx_ch:
                Z[:, 25 * ch:25 * ch + 25] *= -1
            W[:, 0] *= -1
        if flip_y:
            for ch in flipy_ch:
                Z[:, 25 * ch:25 * ch + 25] *= -1
            W[:, 1] *= -1
        outX.append(Z)
        outY.append(W)
    return np.concatenate(outX), np.concatenate(outY)


def train(X, Y, epochs=6, batch=512, lr=1e-3, seed=3, init_seed=1, mirror=True, device=0, form="f64"):
    """Adam on the device from Glorot weights, on the samples and (mirror) their reflections;
    returns (params, mean loss per epoch)."""
    if mirror:
        X, Y = mirrored(X, Y, form)
    return native.learned_train(X, Y, native.learned_init(init_seed), epochs, batch, lr, seed, device)


def unexplained(params, X, Y):
    """Mean squared error of the network's kick over that of no kick (1.0 = no gain)."""
    P = native.learned_predict(X, params)
    return float(np.mean((P - Y) ** 2) / np.mean(Y.astype(np.float64) ** 2))


def zero_network():
    """The network that predicts no kick: the step without the closure's correction."""
    p = np.zeros(native.LEARNED_PARAMS, np.float32)
    p[-1] = 1.0
    return p


def profile(p, x, v):
    """Mean x-velocity per cell row (y bins of one cell)."""
    a_y = p["Ly"] / p["Ny"]
    iy = np.clip((x[1::2] / a_y).astype(int), 0, p["Ny"] - 1)
    n = np.bincount(iy, minlength=p["Ny"])
    return np.bincount(iy, v[0::2], p["Ny"]) / np.maximum(n, 1)


def deploy(p, params, steps, seed=1, every=10, average_from=None, occ_limit=0.0, state=None, bulk_only=True):
    """Runs `steps` steps with the plain closure (params None) or the network; returns the
    time-averaged velocity profile (snapshots every `every` steps from `average_from`), the mean
    occStd and kinetic energy of the metrics rows, and the closure step counts."""
    x, v = state if state is not None else uniform_state(p, seed)
    if average_from is None:
        average_from = steps // 2
    prof = np.zeros(p["Ny"])
    occ, ke, cnt = [], [], 0
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        if params is not None:
            ctx.learned_set(params, occ_limit)
            ctx.learned_options(bulk_only)
        for s0 in range(0, steps, every):
            m = ctx.step(s0, min(every, steps - s0), metrics=True)
            occ.append(m["occStd"])
            ke.append(m["meanKinetic"])
            if s0 + every > average_from:
                xs, vs = ctx.get_state()
                prof += profile(p, xs, vs)
                cnt += 1
        stats = ctx.learned_stats()
    return {"profile": prof / max(cnt, 1), "occStd": float(np.mean(occ)), "meanKinetic": float(np.mean(ke)),
            "closure_steps": stats}


def profile_error(a, b):
    """L2 error of profile a relative to profile b."""
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def time_case(Nx, Ny, ppc, steps, params=None, form="f64"):
    """Device ms per step of the plain and the learned closure on one channel, in one form
    (an untrained Glorot network when params is None: the cost does not depend on the weights)."""
    from .cases import poiseuille_params
    p = poiseuille_params(Nx, Ny, ppc)
    x, v = uniform_state(p, 1)
    if params is None:
        params = native.learned_init(1)
        params[-1] = 0.07
    out = {}
    with native.Context(p, form=form) as ctx:
        ctx.set_state(x, v)
        ctx.step(0, 3)
        out["plain_ms"] = 1e3 * ctx.step_timed(3, steps) / steps
        ctx.learned_set(params)
        ctx.step(3 + steps, 3)
        out["learned_ms"] = 1e3 * ctx.step_timed(6 + steps, steps) / steps
        out["closure_steps"] = ctx.learned_stats()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--runs", type=int, default=200)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--stride", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--out", default="net.npy")
    ap.add_argument("--time-case", type=int, nargs=4, metavar=("NX", "NY", "PPC", "STEPS"),
                    help="only time plain and learned steps on one channel")
    ap.add_argument("--form", choices=["f64", "f32", "fast"], default="f64", help="state form of --time-case")
    a = ap.parse_args()
    if a.time_case:
        print(time_case(*a.time_case, form=a.form))
        return
    t0 = time.time()
    X, Y = collect(a.runs, stride=a.stride, capacity=a.samples, log=print)
    t1 = time.time()
    net, losses = train(X, Y, a.epochs)
    t2 = time.time()
    print(f"{len(X)} samples in {t1 - t0:.1f} s; training {t2 - t1:.1f} s; loss per epoch {losses.tolist()}")
    np.save(a.out, net)


if __name__ == "__main__":
    main()
