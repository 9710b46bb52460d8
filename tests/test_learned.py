"""Learned closure: the network's kernels against the float64 oracle (oracle/mlp_oracle.py), the
dataset collection against the step it samples, and the closure mode switch of the step.

CPU tests pin the oracle itself (finite differences, an independent stencil loop, BF16
rounding against torch). GPU tests call the library through the C-ABI:
- mpcd_learned_predict (the tcgen05 tensor-core kernel) and mpcd_learned_grad against the
  oracle: FP32 accumulation in another order than the oracle's float64 one can move a1 across a
  BF16 rounding boundary (one BF16 ulp, 2^-8 relative, in one of 64 hidden values), so outputs
  agree within 1e-3 of the largest output and to 1e-5 for all but a few rows; gradients within
  1e-4 of the largest entry;
- mpcd_learned_train (one full-batch Adam step) against the oracle's Adam update;
- mpcd_learned_samples: the centre features and targets against the state the step leaves
  (the plain kick is uniform per cell, so the cell mean velocity after the step is the red mean
  plus the target), and every feature against the oracle's stencil of those fields;
- mpcd_learned_set: a zero network gives exactly the step without a closure kick; a learned
  step kicks every particle by the oracle's momentum-conserving kick of its cell (none where
  the stencil crosses a wall); the device
  mode flag follows the occupancy limit, eagerly and under graph replay alike.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as MO  # noqa: E402

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state  # noqa: E402


def _rand_case(rows, seed):
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((rows, MO.FEAT)) * 0.4).astype(np.float32)
    Y = (rng.standard_normal((rows, MO.OUT)) * 0.02).astype(np.float32)
    p = MO.init(seed)
    p[MO.OFF_B1:MO.OFF_W2] = rng.standard_normal(MO.HID) * 0.1
    p[MO.OFF_B3:MO.OFF_SCALE] = rng.standard_normal(MO.OUT) * 0.1
    p[MO.OFF_SCALE] = 0.02
    return X, Y, p


# ---------------------------------------------------------------- the oracle itself (CPU)
def test_oracle_bf16_matches_torch():
    torch = pytest.importorskip("torch")
    a = (np.random.default_rng(1).standard_normal(4096) * 3).astype(np.float32)
    a[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -0.0, 65504.0]  # ties to even both ways
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(MO.bf16(a), ref)


def test_oracle_gradient_finite_differences():
    """The oracle's backward pass against central differences of its loss with the roundings
    held fixed (weights and a1 at their BF16 values): the straight-through gradient."""
    X, Y, p = _rand_case(7, 3)
    loss, g = MO.loss_grad(X, Y, p)
    W = MO.unpack(p)
    rng = np.random.default_rng(4)
    picks = np.concatenate([rng.choice(np.arange(lo, hi), 6, replace=False) for lo, hi in (
        (MO.OFF_W1, MO.OFF_B1), (MO.OFF_B1, MO.OFF_W2), (MO.OFF_W2, MO.OFF_B2), (MO.OFF_B2, MO.OFF_W3),
        (MO.OFF_W3, MO.OFF_B3))] + [np.arange(MO.OFF_B3, MO.OFF_SCALE)])
    flat = np.concatenate([W[0].ravel(), W[1], W[2].ravel(), W[3], W[4].ravel(), W[5]])

    Xr = MO.bf16(X)
    a1_fixed = MO.forward(X, p)[1][2]
    z1_0 = Xr @ W[0].T + W[1]

    def loss_of(q):
        W1 = q[MO.OFF_W1:MO.OFF_B1].reshape(MO.HID, MO.FEAT)
        z1 = Xr @ W1.T + q[MO.OFF_B1:MO.OFF_W2]
        # a1 rounded at the base point, moved by its first-order change (straight through)
        a1 = a1_fixed + (MO.gelu(z1) - MO.gelu(z1_0))
        a2 = MO.gelu(a1 @ q[MO.OFF_W2:MO.OFF_B2].reshape(MO.HID, MO.HID).T + q[MO.OFF_B2:MO.OFF_W3])
        out = a2 @ q[MO.OFF_W3:MO.OFF_B3].reshape(MO.OUT, MO.HID).T + q[MO.OFF_B3:MO.OFF_SCALE]
        e = out - Y.astype(np.float64) / W[6]
        return np.sum(e * e) / e.size

    assert abs(loss_of(flat) - loss) <= 1e-12 * max(1.0, loss)
    h = 1e-6
    for i in picks:
        q1, q2 = flat.copy(), flat.copy()
        q1[i] += h
        q2[i] -= h
        fd = (loss_of(q1) - loss_of(q2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_oracle_stencil_against_loop():
    rng = np.random.default_rng(5)
    Nx, Ny, gamma = 7, 6, 10.0
    N = rng.integers(0, 20, Nx * Ny)
    Ux, Uy = rng.standard_normal(Nx * Ny), rng.standard_normal(Nx * Ny)
    for perx, pery in ((True, False), (False, False), (True, True)):
        F = MO.features(N, Ux, Uy, Nx, Ny, perx, pery, gamma)
        for c in (0, 5, 13, Nx * Ny - 1):
            ix, iy = divmod(c, Ny)
            pts = []
            for dy in range(-2, 3):
                for dx in range(-2, 3):
                    jx, jy = ix + dx, iy + dy
                    ok = True
                    if perx:
                        jx %= Nx
                    elif not 0 <= jx < Nx:
                        ok = False
                    if pery:
                        jy %= Ny
                    elif not 0 <= jy < Ny:
                        ok = False
                    pts.append(jy + Ny * jx if ok else None)
            inside = [q for q in pts if q is not None]
            mx, my = sum(Ux[q] for q in inside) / len(inside), sum(Uy[q] for q in inside) / len(inside)
            for k, q in enumerate(pts):
                want = (N[q] / gamma - 1, Ux[q] - mx, Uy[q] - my) if q is not None else (-1.0, 0.0, 0.0)
                assert np.allclose((F[c, k], F[c, 25 + k], F[c, 50 + k]), want, rtol=0, atol=1e-14), (perx, pery, c, k)


def test_param_layout_matches_header():
    h = open(os.path.join(ROOT, "include", "mpcd_c.h")).read()
    assert f"#define MPCD_LEARNED_PARAMS {MO.N_PARAMS}" in h
    assert f"#define MPCD_LEARNED_FEATURES {MO.FEAT}" in h
    assert f"#define MPCD_LEARNED_OUTPUTS {MO.OUT}" in h


# ---------------------------------------------------------------- kernels on the GPU
def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no CUDA device")
    return native


@pytest.mark.gpu
def test_predict_matches_oracle():
    native = _native()
    X, _, p = _rand_case(1000, 11)  # 7 full tiles of 128 rows and a partial one
    got = native.learned_predict(X, p)
    want = MO.predict(X, p)
    top = np.max(np.abs(want))
    err = np.max(np.abs(got - want), axis=1)
    assert np.max(err) <= 1e-3 * top
    assert np.count_nonzero(err > 1e-5 * top) <= 10


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [1, 16, 100, 1000])
def test_gradient_matches_oracle(rows):
    native = _native()
    X, Y, p = _rand_case(rows, 20 + rows)
    g, loss = native.learned_grad(X, Y, p)
    loss_o, g_o = MO.loss_grad_tc(X, Y, p)  # the tensor-core kernel's BF16 backward operands
    assert abs(loss - loss_o) <= 1e-5 * loss_o
    assert g[MO.OFF_SCALE] == 0.0
    scale = np.max(np.abs(g_o))
    for lo, hi in ((MO.OFF_W1, MO.OFF_B1), (MO.OFF_B1, MO.OFF_W2), (MO.OFF_W2, MO.OFF_B2), (MO.OFF_B2, MO.OFF_W3),
                   (MO.OFF_W3, MO.OFF_B3), (MO.OFF_B3, MO.OFF_SCALE)):
        assert np.max(np.abs(g[lo:hi] - g_o[lo:hi])) <= 1e-4 * scale, (rows, lo)


@pytest.mark.gpu
def test_adam_step_matches_oracle():
    """One epoch with one batch holding every row = one Adam step from zero moments."""
    native = _native()
    X, Y, p = _rand_case(64, 31)
    lr = 1e-3
    q, losses = native.learned_train(X, Y, p, epochs=1, batch=64, lr=lr, seed=1)
    loss_o, g_o = MO.loss_grad_tc(X, Y, p)
    assert abs(losses[0] - loss_o) <= 1e-5 * loss_o
    want, _, _ = MO.adam_step(p, g_o, np.zeros_like(g_o), np.zeros_like(g_o), 1, lr)
    big = np.abs(g_o) > 1e-3 * np.max(np.abs(g_o))  # g / (|g| + eps) is ill-conditioned near 0
    big[MO.OFF_SCALE] = False
    assert np.max(np.abs(q[big] - want[big])) <= 1e-6
    assert q[MO.OFF_SCALE] == p[MO.OFF_SCALE]
    assert np.all(np.abs(q[:MO.OFF_SCALE] - p[:MO.OFF_SCALE]) <= lr * 1.0001)


@pytest.mark.gpu
def test_training_lowers_loss():
    native = _native()
    rng = np.random.default_rng(7)
    X = (rng.standard_normal((4096, MO.FEAT)) * 0.3).astype(np.float32)
    Y = np.stack([X[:, 12] - X[:, 13], X[:, 37] * X[:, 62]], 1).astype(np.float32) * 0.01
    p = native.learned_init(3)
    q, losses = native.learned_train(X, Y, p, epochs=8, batch=128, lr=2e-3, seed=2)
    assert q[MO.OFF_SCALE] > 0
    assert losses[-1] < 0.2 * losses[0], losses


def _cells(p, x, v):
    a_x, a_y = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
    xy = x.reshape(-1, 2)
    ix = np.clip(np.floor(xy[:, 0] / a_x).astype(int), 0, p["Nx"] - 1)
    iy = np.clip(np.floor(xy[:, 1] / a_y).astype(int), 0, p["Ny"] - 1)
    c = iy + p["Ny"] * ix
    N = np.bincount(c, minlength=p["Nc"])
    vv = v.reshape(-1, 2)
    sx = np.bincount(c, vv[:, 0], p["Nc"])
    sy = np.bincount(c, vv[:, 1], p["Nc"])
    with np.errstate(invalid="ignore", divide="ignore"):
        return N, np.where(N > 0, sx / np.maximum(N, 1), 0.0), np.where(N > 0, sy / np.maximum(N, 1), 0.0)


@pytest.mark.gpu
def test_samples_match_the_step():
    native = _native()
    p = poiseuille_params(40, 20, 10)
    x, v = uniform_state(p, 9)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.step(0, 3)
        X, Y = ctx.learned_samples(3, 2, stride=1)
        assert X.shape == (2 * p["Nc"], 75) and Y.shape == (2 * p["Nc"], 2)
        xs, vs = ctx.get_state()
    X, Y = X[p["Nc"]:], Y[p["Nc"]:]  # the last step's rows, every cell in order
    N, Ux, Uy = _cells(p, xs, vs)
    assert np.array_equal(X[:, 12], (N / p["gamma"] - 1).astype(np.float32))
    red_ux, red_uy = Ux - Y[:, 0], Uy - Y[:, 1]  # the plain kick is uniform per cell
    F = MO.features(N, red_ux, red_uy, p["Nx"], p["Ny"], True, False, p["gamma"])  # channel: periodic x, walls in y
    assert np.max(np.abs(X - F)) <= 2e-6
    assert np.max(np.abs(Y)) > 0


def _phases_without_closure(ctx, s):
    ctx.stream()
    ctx.apply_bc(104729 + 10007 * s)
    ctx.srd_shift_cells(130363 + 10007 * s, want_cells=False)
    ctx.srd_collide(433494437 + 10007 * s)
    ctx.save_ref()
    ctx.zone_pass("base", 88172645463325252 + 10007 * s)
    ctx.zone_pass("shifted", 88172645463325252 + 4099 + 10007 * s)


@pytest.mark.gpu
def test_zero_network_is_the_step_without_kick():
    native = _native()
    p = poiseuille_params(40, 20, 10)
    x, v = uniform_state(p, 12)
    zero = np.zeros(native.LEARNED_PARAMS, np.float32)
    zero[MO.OFF_SCALE] = 1.0
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.learned_set(zero)
        ctx.step(0, 1)
        xl, vl = ctx.get_state()
        assert ctx.learned_stats() == (0, 1, 1)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        _phases_without_closure(ctx, 1)
        xp, vp = ctx.get_state()
    assert np.array_equal(xl, xp)
    assert np.array_equal(vl, vp)


@pytest.mark.gpu
def test_learned_kick_matches_oracle():
    """A learned step = the step without closure kick, then every particle of cell c kicked by
    the network's output on the stencil of the red fields (the tensor-core kernel in the step)."""
    native = _native()
    p = poiseuille_params(48, 24, 10)
    x, v = uniform_state(p, 15)
    net = native.learned_init(8)
    net[MO.OFF_B1:MO.OFF_W2] = np.random.default_rng(2).standard_normal(MO.HID) * 0.2
    net[MO.OFF_SCALE] = 1e-2
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.learned_set(net)
        ctx.step(0, 1)
        xl, vl = ctx.get_state()
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        _phases_without_closure(ctx, 1)
        xr, vr = ctx.get_state()
    assert np.array_equal(xl, xr)
    N, Ux, Uy = _cells(p, xr, vr)
    F = MO.features(N, Ux, Uy, p["Nx"], p["Ny"], True, False, p["gamma"])
    bulk = MO.bulk_mask(p["Nx"], p["Ny"], True, False)
    want = MO.conserving(MO.predict(F.astype(np.float32), net) * bulk[:, None], N)
    a_x, a_y = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
    c = (np.floor(xr[1::2] / a_y).astype(int).clip(0, p["Ny"] - 1) +
         p["Ny"] * np.floor(xr[0::2] / a_x).astype(int).clip(0, p["Nx"] - 1))
    kick = (vl - vr).reshape(-1, 2)
    # momentum: only the int64 rounding of each cell's N du (2^-33 at most) survives
    assert np.all(np.abs(kick.sum(0)) <= p["Nc"] * 2.0 ** -33 + 1e-10)
    top = np.max(np.abs(want))
    err = np.abs(kick - want[c]).max(axis=1)
    assert np.max(err) <= 1e-3 * top + 1e-12
    assert np.count_nonzero(err > 1e-5 * top + 1e-12) <= 0.01 * len(err)


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_mode_switch_follows_occupancy_limit(graphs):
    native = _native()
    p = poiseuille_params(40, 20, 10)
    x, v = uniform_state(p, 13)
    net = native.learned_init(5)
    net[MO.OFF_SCALE] = 1e-3
    out = {}
    for limit, want in ((0.0, (0, 6, 1)), (1e-9, (5, 1, 0)), (1e9, (0, 6, 1))):
        with native.Context(p) as ctx:
            ctx.set_graphs(graphs)
            ctx.set_state(x, v)
            ctx.learned_set(net, limit)
            ctx.step(0, 6)
            assert ctx.learned_stats() == want, limit
            out[limit] = ctx.get_state()
            ctx.learned_set(None)
            ctx.step(6, 2)
            assert ctx.learned_stats()[:2] == want[:2]  # unset: plain steps, counters frozen
    assert np.array_equal(out[0.0][1], out[1e9][1])
    assert not np.array_equal(out[0.0][1], out[1e-9][1])


@pytest.mark.gpu
def test_graph_replay_matches_eager_with_network():
    native = _native()
    p = poiseuille_params(40, 20, 10)
    x, v = uniform_state(p, 14)
    net = native.learned_init(6)
    net[MO.OFF_SCALE] = 1e-3
    res = []
    for graphs in (True, False):
        with native.Context(p) as ctx:
            ctx.set_graphs(graphs)
            ctx.set_state(x, v)
            ctx.learned_set(net, 0.35)
            ctx.step(0, 8)
            res.append((ctx.get_state(), ctx.learned_stats()))
    assert res[0][1] == res[1][1]
    assert np.array_equal(res[0][0][0], res[1][0][0]) and np.array_equal(res[0][0][1], res[1][0][1])


@pytest.mark.gpu
def test_network_gain_over_no_kick():
    """What the trained network gains over the method without it. The network is trained on
    samples of 12 channels of the ensemble family and scored on 2 held-out channels: its kick
    must explain a share of the plain closure's kick (no kick explains none). In deployment on
    an unseen channel it must keep the plain closure's statistics (kinetic energy, occupancy
    spread) and take every step itself."""
    from src_incompressible_openmp_b200 import learned as L
    X, Y = L.collect(runs=12, seed=21, warmup=40, steps=10, stride=3)
    net, losses = L.train(X, Y, epochs=4)
    assert losses[-1] < losses[0]
    Xh, Yh = L.collect(runs=2, seed=99, warmup=40, steps=5, stride=3)
    fvu = L.unexplained(net, Xh, Yh)
    assert fvu < 0.85, fvu
    assert L.unexplained(L.zero_network(), Xh, Yh) == pytest.approx(1.0)
    p = poiseuille_params(128, 64, 10)
    plain = L.deploy(p, None, 300)
    lrn = L.deploy(p, net, 300)
    assert lrn["closure_steps"] == (0, 300, 1)
    assert abs(lrn["meanKinetic"] / plain["meanKinetic"] - 1) < 0.02
    assert abs(lrn["occStd"] / plain["occStd"] - 1) < 0.05
