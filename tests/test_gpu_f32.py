"""The FP32 precision form (mpcd_ctx_create_form(..., MPCD_FORM_F32)) against the FP64 plain form.

The FP32 form stores per particle the standard-grid cell, the FP32 offset inside the cell and
FP32 velocities; the arithmetic of every kernel is the plain form's, in FP64 registers. So:
- state I/O rounds a state exactly as the form defines: offsets to FP32 relative to the cell,
  velocities to FP32;
- one step from an FP32-representable state follows the plain step closely: the per-store
  roundings (2^-24 relative) move a few particles across redistribution decisions, which the
  test bounds, and leave cell occupancies and the particle count exact;
- over many steps the runs decorrelate (the dynamics is chaotic), so the statistics are compared:
  kinetic energy, occupancy spread and the time-averaged velocity profile against the plain
  run, within the spread between two plain runs of different seeds;
- graph replay equals eager steps bit for bit, and the learned closure runs on the FP32 state.
"""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no CUDA device")
    return native


def _f32_state(p, x, v):
    """The state as the FP32 form stores it (cell, FP32 offset, FP32 velocity), widened."""
    dx, dy = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
    X = x.reshape(-1, 2)
    ix = np.clip(np.floor(X[:, 0] / dx).astype(int), 0, p["Nx"] - 1)
    iy = np.clip(np.floor(X[:, 1] / dy).astype(int), 0, p["Ny"] - 1)
    ox = (X[:, 0] - ix * dx).astype(np.float32).astype(np.float64)
    oy = (X[:, 1] - iy * dy).astype(np.float32).astype(np.float64)
    xr = np.stack([ix * dx + ox, iy * dy + oy], 1).reshape(-1)
    return xr, v.astype(np.float32).astype(np.float64)


def test_state_io_rounds_as_defined():
    native = _native()
    p = poiseuille_params(64, 32, 10)
    x, v = uniform_state(p, 3)
    with native.Context(p, form="f32") as ctx:
        ctx.set_state(x, v)
        xg, vg = ctx.get_state()
    xr, vr = _f32_state(p, x, v)
    assert np.array_equal(vg, vr)
    assert np.max(np.abs(xg - xr)) <= 1e-15 * p["Lx"]
    assert np.max(np.abs(xg - x)) <= 2.0 ** -24 * p["Lx"] / p["Nx"]


def test_phase_functions_rejected():
    native = _native()
    p = poiseuille_params(16, 16, 5)
    x, v = uniform_state(p, 1)
    with native.Context(p, form="f32") as ctx:
        ctx.set_state(x, v)
        with pytest.raises(native.MpcdError):
            ctx.stream()
        with pytest.raises(native.MpcdError):
            ctx.zone_pass("base", 1)


def test_one_step_follows_plain():
    native = _native()
    p = poiseuille_params(96, 48, 10)
    x, v = uniform_state(p, 4)
    x, v = _f32_state(p, x, v)  # both forms start from the same representable state
    out = {}
    for form in ("f64", "f32"):
        with native.Context(p, form=form) as ctx:
            ctx.set_state(x, v)
            m = ctx.step(0, 1, metrics=True)
            out[form] = (*ctx.get_state(), m)
    x64, v64, m64 = out["f64"]
    x32, v32, m32 = out["f32"]
    dx = p["Lx"] / p["Nx"]
    moved = np.any(np.abs(x32 - x64).reshape(-1, 2) > 1e-6 * dx, axis=1)
    assert np.count_nonzero(moved) <= 0.01 * p["n"]
    same = ~moved
    assert np.max(np.abs(x32 - x64).reshape(-1, 2)[same]) <= 1e-6 * dx
    dv = np.abs(v32 - v64).reshape(-1, 2)[same]
    assert np.quantile(dv, 0.99) <= 1e-5
    assert abs(m32["meanKinetic"] / m64["meanKinetic"] - 1) <= 1e-4
    assert m32["shiftedOutBand"] == pytest.approx(m64["shiftedOutBand"], abs=0.01)


def _profile(p, x, v):
    a_y = p["Ly"] / p["Ny"]
    iy = np.clip((x[1::2] / a_y).astype(int), 0, p["Ny"] - 1)
    return np.bincount(iy, v[0::2], p["Ny"]) / np.maximum(np.bincount(iy, minlength=p["Ny"]), 1)


def _run(native, p, form, seed, steps=600, every=20):
    x, v = uniform_state(p, seed)
    ke, occ, prof, cnt = [], [], np.zeros(p["Ny"]), 0
    with native.Context(p, form=form) as ctx:
        ctx.set_state(x, v)
        for s0 in range(0, steps, every):
            m = ctx.step(s0, every, metrics=True)
            ke.append(m["meanKinetic"])
            occ.append(m["occStd"])
            if s0 >= steps // 2:
                xs, vs = ctx.get_state()
                prof += _profile(p, xs, vs)
                cnt += 1
    return np.mean(ke), np.mean(occ), prof / cnt


def test_statistics_match_plain():
    native = _native()
    p = poiseuille_params(256, 64, 10)
    k64, o64, p64 = _run(native, p, "f64", 1)
    k32, o32, p32 = _run(native, p, "f32", 1)
    kb, ob, pb = _run(native, p, "f64", 2)  # the plain form's own seed-to-seed spread
    floor = np.linalg.norm(pb - p64) / np.linalg.norm(p64)
    err = np.linalg.norm(p32 - p64) / np.linalg.norm(p64)
    assert err <= 2.0 * floor + 0.01, (err, floor)
    assert abs(k32 / k64 - 1) <= 2.0 * abs(kb / k64 - 1) + 2e-3
    assert abs(o32 / o64 - 1) <= 2.0 * abs(ob / o64 - 1) + 5e-3


def test_graph_replay_matches_eager():
    native = _native()
    p = poiseuille_params(64, 32, 10)
    x, v = uniform_state(p, 6)
    res = []
    for graphs in (True, False):
        with native.Context(p, form="f32") as ctx:
            ctx.set_graphs(graphs)
            ctx.set_state(x, v)
            ctx.step(0, 8)
            res.append(ctx.get_state())
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_learned_closure_on_f32_state():
    native = _native()
    p = poiseuille_params(64, 32, 10)
    x, v = uniform_state(p, 7)
    net = native.learned_init(2)
    net[-1] = 1e-3
    with native.Context(p, form="f32") as ctx:
        ctx.set_state(x, v)
        X, Y = ctx.learned_samples(0, 2, 3)
        assert len(X) > 0 and np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
        ctx.learned_set(net)
        ctx.step(2, 5)
        assert ctx.learned_stats() == (0, 5, 1)
        xs, vs = ctx.get_state()
    assert np.all(np.isfinite(xs)) and np.all(np.isfinite(vs))
