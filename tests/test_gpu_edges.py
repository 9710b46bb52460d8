"""Edge cases of the CUDA path against the oracle, through the C-ABI:

- clump: a dense blob (hundreds of particles per cell) forces cell segments longer than 32
  (the index's insertion-sort path), shuffles of more than 32 entries (the sequential path),
  and zones whose lists outgrow the shared-memory arena (the global-memory overflow kernel);
- high density: 40 particles per cell everywhere;
- tiny periodic: a 4x3 domain periodic in both axes, smaller than one zone tile, where
  range-2 neighbour offsets wrap onto the same cell;
- no particles at all;
- an unsupported wall mode, which fails only once a particle crosses that wall;
- positions on cell and period boundaries and one ulp either side, where the kernels' floor
  of x / dx (a multiply by the reciprocal, certified, else a division) must take the division.
Bars as in test_gpu_parity: positions, counts and moves bit-exact; velocities within 1e-12
relative per step.
"""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu

REL = 1e-12


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def vclose(a, b):
    d = np.abs(a - b) / np.maximum(1.0, np.abs(b))
    return float(d.max()) if d.size else 0.0


def clump_state(p, seed, frac=0.4, cells=3):
    """Uniform state with a fraction of the particles packed into a cells x cells blob."""
    x, v = uniform_state(p, seed)
    rng = np.random.default_rng(seed + 1)
    n = p["n"]
    k = int(frac * n)
    a = p["Lx"] / p["Nx"]
    x = x.reshape(-1, 2)
    x[:k, 0] = p["Lx"] * 0.5 + a * cells * (rng.random(k) - 0.5)
    x[:k, 1] = p["Ly"] * 0.5 + a * cells * (rng.random(k) - 0.5)
    return x.reshape(-1).copy(), v


def run_steps_both(native, oracle, p, x, v, nsteps):
    """Teacher-forced steps: GPU and oracle from the same input at every step."""
    with native.Context(p) as ctx:
        xo, vo = x, v
        for s in range(1, nsteps + 1):
            ctx.set_state(xo, vo)
            m = ctx.step(s - 1, 1, metrics=True)
            xg, vg = ctx.get_state()
            xo, vo, mo = oracle.step(p, xo, vo, s)
            assert np.array_equal(xg, xo), f"step {s} positions"
            assert vclose(vg, vo) <= REL, f"step {s} velocities"
            for ph in ("base", "shifted"):
                assert m[ph]["nParticlesMovedDense"] == mo[ph]["nParticlesMovedDense"], (s, ph)
                assert m[ph]["nParticlesMovedSparse"] == mo[ph]["nParticlesMovedSparse"], (s, ph)


def test_clump_overflow_paths(oracle):
    native = _native()
    p = poiseuille_params(30, 20, 10)
    x, v = clump_state(p, 61)
    # the blob holds ~270 particles per cell: check that the case exercises what it claims
    cid = (np.floor(x[0::2] / (p["Lx"] / p["Nx"])).astype(int) * p["Ny"] +
           np.floor(x[1::2] / (p["Ly"] / p["Ny"])).astype(int))
    assert np.bincount(cid).max() > 64
    run_steps_both(native, oracle, p, x, v, 3)
    # zone pass phase by phase (the pass sees the blob at full height)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.save_ref()
        for mode, seed in (("base", 88172645463325252 + 10007 * 3), ("shifted", 88172645463325252 + 4099 + 10007 * 3)):
            xin, vin = ctx.get_state()
            mg = ctx.zone_pass(mode, seed)
            xo, vo, mo = oracle.zone_pass(p, xin, vin, mode, seed)
            xg, vg = ctx.get_state()
            assert np.array_equal(xg, xo) and np.array_equal(vg, vo), mode
            assert mg["nParticlesMovedDense"] == mo["nParticlesMovedDense"], mode


def test_high_density(oracle):
    native = _native()
    p = poiseuille_params(20, 12, 40)
    x, v = uniform_state(p, 62)
    run_steps_both(native, oracle, p, x, v, 2)


def test_tiny_periodic_domain(oracle):
    native = _native()
    p = poiseuille_params(4, 3, 12, boundary_bottom="periodic", boundary_top="periodic", g=0.01)
    x, v = uniform_state(p, 63)
    run_steps_both(native, oracle, p, x, v, 3)


def test_no_particles(oracle):
    native = _native()
    p = poiseuille_params(16, 8, 10)
    p["n"] = 0
    x = np.zeros(0)
    v = np.zeros(0)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.step(0, 2)
        xg, vg = ctx.get_state()
        f = ctx.cell_fields(1.0)
    assert xg.size == 0 and vg.size == 0
    assert not f["N"].any()
    xo, vo, _ = oracle.step(p, x, v, 1)
    assert xo.size == 0 and vo.size == 0


def test_unsupported_wall_mode_fails_on_crossing(oracle):
    native = _native()
    p = poiseuille_params(12, 8, 10, boundary_bottom="sticky")
    x, v = uniform_state(p, 64)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.stream()
        with pytest.raises(native.MpcdError) as e:
            ctx.apply_bc(104729)
        assert e.value.code == 3 and "boundary_bottom" in str(e.value)
    xs, vs = oracle.stream(p, x, v)
    with pytest.raises(Exception):
        oracle.apply_bc(p, xs, vs, 104729)


def boundary_state(p, seed):
    """Uniform state whose positions are moved onto cell and period boundaries: k dx exactly
    (as rounded), the neighbouring doubles, 0, Lx and the double below Lx."""
    x, v = uniform_state(p, seed)
    rng = np.random.default_rng(seed + 7)
    X = x.reshape(-1, 2)
    n = len(X)
    dx, dy = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
    kx = rng.integers(0, p["Nx"] + 1, n)
    ky = rng.integers(1, p["Ny"], n)
    bx = kx * dx
    by = ky * dy
    which = rng.integers(0, 4, n)
    bx = np.where(which == 1, np.nextafter(bx, -np.inf), np.where(which == 2, np.nextafter(bx, np.inf), bx))
    by = np.where(which == 3, np.nextafter(by, np.inf), np.where(which == 1, np.nextafter(by, -np.inf), by))
    pick = rng.random(n) < 0.5
    X[pick, 0] = np.clip(bx[pick], 0.0, np.nextafter(p["Lx"], 0.0))
    X[pick, 1] = by[pick]
    X[:4, 0] = [0.0, np.nextafter(p["Lx"], 0.0), p["Lx"] * 0.5, np.nextafter(0.0, 1.0)]
    return X.reshape(-1).copy(), v


def test_positions_on_cell_boundaries(oracle):
    native = _native()
    p = poiseuille_params(64, 32, 8)
    x, v = boundary_state(p, 81)
    rho_t = p["gamma"] / ((p["Lx"] / p["Nx"]) * (p["Ly"] / p["Ny"]))
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        fg = ctx.cell_fields(rho_t)
        fo = oracle.cell_fields(p, x, v, rho_t)
        assert np.array_equal(fg["N"], fo["N"]), "cell counts"
        for seed in (5, 130363, 991):
            assert np.array_equal(ctx.srd_shift_cells(seed), oracle.srd_shift_cells(p, x, seed)), seed
    run_steps_both(native, oracle, p, x, v, 3)


def test_single_full_domain_graph_replay_matches_eager():
    """With the single full-domain zone, the second pass of a step still takes the shifted
    pass's seed (seedBase + 4099), in eager steps and in graph replays alike."""
    native = _native()
    p = poiseuille_params(16, 12, 10, zoneSingleFullDomainMode=True)
    x, v = uniform_state(p, 91)
    res = []
    for graphs in (True, False):
        with native.Context(p) as ctx:
            ctx.set_graphs(graphs)
            ctx.set_state(x, v)
            ctx.step(0, 6)
            res.append(ctx.get_state())
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
