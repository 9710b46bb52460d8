"""The fast form (MPCD_FORM_FAST): FP32 bins, counter-based draws, order-free redistribution.

It does not follow the reference's draws, so it is not compared particle by particle with the
oracle. It is held to what it promises instead:
  - state I/O: positions round to FP32 offsets inside their cell, velocities to the 2^-20 grid;
    no particle is lost or duplicated by a step (a missing particle would read back as NaN);
  - order-free: the same input gives bit-identical output in particle-id order, in separate
    contexts (the order of particles inside the bins comes from atomics and differs);
  - conservation: with the closure kick, the body force and the walls switched off
    (periodic box), total momentum is kept exactly, to the last 2^-20 unit, over many steps
    (collision and both zone passes conserve it);
  - physics: on a Poiseuille channel the time-averaged velocity profile, kinetic energy and
    occupancy spread agree with the plain FP64 form within the plain form's own seed-to-seed
    spread.
"""
import os

import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu

Q = 2.0 ** 20


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def test_state_round_trip():
    native = _native()
    p = poiseuille_params(48, 32, 10)
    x, v = uniform_state(p, 3)
    with native.Context(p, form="fast") as ctx:
        ctx.set_state(x, v)
        xg, vg = ctx.get_state()
    assert np.array_equal(vg, np.round(v * Q) / Q)
    a = p["Lx"] / p["Nx"]
    assert np.max(np.abs(xg - x)) <= a * 2.0 ** -23
    assert not np.isnan(xg).any()


def test_step_keeps_every_particle_and_is_order_free():
    native = _native()
    p = poiseuille_params(64, 40, 12)
    x, v = uniform_state(p, 4)
    out = []
    for _ in range(2):
        with native.Context(p, form="fast") as ctx:
            ctx.set_state(x, v)
            m = ctx.step(0, 8, metrics=True)
            out.append(ctx.get_state())
            assert m["base"]["nParticlesMovedDense"] + m["base"]["nParticlesMovedSparse"] > 0
    (x1, v1), (x2, v2) = out
    assert not np.isnan(x1).any() and not np.isnan(v1).any()
    assert np.all((x1[0::2] >= 0) & (x1[0::2] <= p["Lx"])) and np.all((x1[1::2] >= 0) & (x1[1::2] <= p["Ly"]))
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    # velocities stay on the grid
    assert np.array_equal(v1 * Q, np.round(v1 * Q))


def test_momentum_exact_without_kicks():
    native = _native()
    p = poiseuille_params(60, 40, 20, boundary_bottom="periodic", boundary_top="periodic", bodyForceX=0.0,
                          betaEOS=0.0, betaRepair=0.0, useOptimalBetaRepair=False)
    x, v = uniform_state(p, 5)
    with native.Context(p, form="fast") as ctx:
        ctx.set_state(x, v)
        _, v0 = ctx.get_state()
        P0 = np.round(v0 * Q).astype(np.int64).reshape(-1, 2).sum(axis=0)
        moved = 0
        for k in range(5):
            m = ctx.step(4 * k, 4, metrics=True)
            moved += sum(m[ph][f] for ph in ("base", "shifted") for f in ("nParticlesMovedDense", "nParticlesMovedSparse"))
            _, vk = ctx.get_state()
            Pk = np.round(vk * Q).astype(np.int64).reshape(-1, 2).sum(axis=0)
            assert np.array_equal(Pk, P0), (k, Pk - P0)
    assert moved > 0


def test_collision_spill_path_matches_tiles():
    """SRD tiles whose standard cells hold more particles than the tile kernel's shared memory
    are collided by the spill kernel; sending every tile there gives the same state."""
    native = _native()
    p = poiseuille_params(70, 45, 12)
    x, v = uniform_state(p, 6)
    out = []
    for pcap in (None, "64"):
        if pcap:
            os.environ["MPCD_FAST_COLLIDE_PCAP"] = pcap
        try:
            with native.Context(p, form="fast") as ctx:
                ctx.set_state(x, v)
                ctx.step(0, 6)
                out.append(ctx.get_state())
        finally:
            os.environ.pop("MPCD_FAST_COLLIDE_PCAP", None)
    (x1, v1), (x2, v2) = out
    assert not np.isnan(v1).any()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)


def test_autotuners_leave_state_unchanged(monkeypatch):
    """The collision's autotuner times every tile height on the live state and restores it, and
    the zone autotuner runs the first base pass's decisions with 8 and 4 zones per block (both
    at the first step): the run, and the first step's move counters, equal a run without
    tuning, bit for bit."""
    native = _native()
    p = poiseuille_params(64, 40, 20)
    x, v = uniform_state(p, 9)
    out = []
    for tune in (True, False):
        monkeypatch.setenv("MPCD_FAST_COLLIDE_TUNE", "1" if tune else "0")
        if tune:
            monkeypatch.delenv("MPCD_FAST_ZONE_WARPS", raising=False)
        else:
            monkeypatch.setenv("MPCD_FAST_ZONE_WARPS", "8")
        with native.Context(p, form="fast") as ctx:
            ctx.set_state(x, v)
            m1 = ctx.step(0, 1, metrics=True)
            ctx.step(1, 3)
            out.append((ctx.get_state(), m1))
    ((x1, v1), m1), ((x2, v2), m2) = out
    assert not np.isnan(v1).any()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert m1["base"] == m2["base"] and m1["shifted"] == m2["shifted"]


def _profile(native, p, seed, form, steps, avg_from):
    x, v = uniform_state(p, seed)
    with native.Context(p, form=form) as ctx:
        ctx.set_state(x, v)
        ctx.step(0, avg_from)
        ctx.profile_reset(True)
        m = ctx.step(avg_from, steps - avg_from, metrics=True)
        ux, k = ctx.profile_read()
    assert k == steps - avg_from
    return ux, m


def test_channel_statistics_match_plain_form():
    """256 x 64 channel, 10 per cell, 1200 steps, profile averaged over steps 400-1200."""
    native = _native()
    p = poiseuille_params(256, 64, 10)
    steps, avg_from = 1200, 400
    plain1, m1 = _profile(native, p, 11, "f64", steps, avg_from)
    plain2, m2 = _profile(native, p, 12, "f64", steps, avg_from)
    fast, mf = _profile(native, p, 11, "fast", steps, avg_from)
    norm = np.linalg.norm(plain1)
    noise = np.linalg.norm(plain2 - plain1) / norm
    err = np.linalg.norm(fast - plain1) / norm
    assert err <= max(2.0 * noise, 0.02), (err, noise)
    ke_noise = abs(m2["meanKinetic"] - m1["meanKinetic"])
    assert abs(mf["meanKinetic"] - m1["meanKinetic"]) <= max(3 * ke_noise, 0.01 * m1["meanKinetic"])
    assert mf["occStd"] <= 2.0 * max(m1["occStd"], m2["occStd"])


def test_learned_eos_kick_network_gain():
    """The fast form's network (the EOS kick from the collided state's stencil) trained on 12
    channels of the ensemble family explains most of the plain EOS kick on 2 held-out channels
    (no kick explains none); deployed, it takes every step itself and keeps the plain closure's
    kinetic energy and occupancy spread."""
    native = _native()
    from src_incompressible_openmp_b200 import learned as L
    X, Y = L.collect(runs=12, seed=21, warmup=40, steps=10, stride=3, form="fast")
    net, losses = L.train(X, Y, epochs=4, form="fast")
    assert losses[-1] < 0.1 * losses[0], losses
    Xh, Yh = L.collect(runs=2, seed=99, warmup=40, steps=5, stride=3, form="fast")
    fvu = L.unexplained(net, Xh, Yh)
    assert fvu < 0.2, fvu
    assert L.unexplained(L.zero_network(), Xh, Yh) == pytest.approx(1.0)
    p = poiseuille_params(512, 128, 20)
    x, v = uniform_state(p, 1)
    rows = {}
    for name, params in (("plain", None), ("learned", net)):
        with native.Context(p, form="fast") as ctx:
            ctx.set_state(x, v)
            if params is not None:
                ctx.learned_set(params, 10.0)
            ctx.step(0, 300)
            rows[name] = ctx.step(300, 300, metrics=True)
            if params is not None:
                plain_steps, learned_steps, _ = ctx.learned_stats()
                assert plain_steps == 0 and learned_steps == 600
    assert abs(rows["learned"]["meanKinetic"] / rows["plain"]["meanKinetic"] - 1) < 0.02
    assert abs(rows["learned"]["occStd"] / rows["plain"]["occStd"] - 1) < 0.05

