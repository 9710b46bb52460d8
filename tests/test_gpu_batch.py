"""Batched replicas (mpcd_batch_*) and graph replay: replicas of different sizes and forcing,
advanced together, give exactly what each gives alone, with and without CUDA-graph replay,
and track the oracle."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu

REPLICAS = [
    (dict(Nx=40, Ny=20, ppc=10), "uniform", 51),
    (dict(Nx=24, Ny=16, ppc=8, bodyForceX=3e-3, g=0.002), "uniform", 52),
    (dict(Nx=30, Ny=30, ppc=12, bodyForceX=2e-4), "checker", 53),
]


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def _case(over, kind, seed):
    over = dict(over)
    Nx, Ny, ppc = over.pop("Nx"), over.pop("Ny"), over.pop("ppc")
    p = poiseuille_params(Nx, Ny, ppc, **over)
    x, v = uniform_state(p, seed) if kind == "uniform" else modulated_state(p, seed, mode=kind)
    return p, x, v


def test_batch_equals_replicas_alone(oracle):
    native = _native()
    cases = [_case(*r) for r in REPLICAS]
    nsteps = 5
    alone = []
    for graphs in (True, False):
        outs = []
        for p, x, v in cases:
            with native.Context(p) as ctx:
                ctx.set_graphs(graphs)
                ctx.set_state(x, v)
                ctx.step(0, nsteps)
                outs.append(ctx.get_state())
        alone.append(outs)
    for (xa, va), (xb, vb) in zip(*alone):  # graph replay = eager steps, bit for bit
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    # batched steps (the zone kernels of all replicas in one launch per pass), replayed from
    # the batch's graph after the first step, or eager when a member has graphs off
    for graphs in (True, False):
        with native.Batch([c[0] for c in cases]) as B:
            for i, (p, x, v) in enumerate(cases):
                B.member(i).set_state(x, v)
                B.member(i).set_graphs(graphs)
            t = B.step(0, 2)
            t += B.step(2, nsteps - 2)
            assert t > 0.0
            for i in range(len(cases)):
                xg, vg = B.member(i).get_state()
                assert np.array_equal(xg, alone[0][i][0]) and np.array_equal(vg, alone[0][i][1]), (graphs, i)
    # the first replica against the oracle (free run: one-ulp thermal draws may propagate)
    p, x, v = cases[0]
    xo, vo = x, v
    for s in range(1, nsteps + 1):
        xo, vo, _ = oracle.step(p, xo, vo, s)
    rel = lambda a, b: float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))
    assert rel(alone[0][0][0], xo) <= 1e-9 and rel(alone[0][0][1], vo) <= 1e-9


def _alone(native, p, x, v, step0, nsteps):
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.step(step0, nsteps)
        return ctx.get_state()


def test_batch_index_fallbacks():
    """The replicas' cell indexes are built by one launch per kernel when every replica fits
    the one-block scan (Nc <= 65,536) and all share a particle-id buffer parity; otherwise each
    replica builds its own. Both give the replicas' results alone."""
    native = _native()
    big = _case(dict(Nx=320, Ny=240, ppc=2), "uniform", 61)  # 76,800 cells: per-replica builds
    small = _case(dict(Nx=32, Ny=16, ppc=9), "uniform", 62)
    with native.Batch([big[0], small[0]]) as B:
        for i, (p, x, v) in enumerate((big, small)):
            B.member(i).set_state(x, v)
        B.step(0, 3)
        for i, (p, x, v) in enumerate((big, small)):
            xg, vg = B.member(i).get_state()
            xa, va = _alone(native, p, x, v, 0, 3)
            assert np.array_equal(xg, xa) and np.array_equal(vg, va), i
    # parities differ after one member's state is uploaded again mid-run
    other = _case(dict(Nx=28, Ny=20, ppc=7), "uniform", 63)
    x2, v2 = uniform_state(other[0], 64)
    with native.Batch([small[0], other[0]]) as B:
        B.member(0).set_state(small[1], small[2])
        B.member(1).set_state(other[1], other[2])
        B.step(0, 1)
        B.member(1).set_state(x2, v2)
        B.step(1, 3)
        xg, vg = B.member(0).get_state()
        xa, va = _alone(native, small[0], small[1], small[2], 0, 4)
        assert np.array_equal(xg, xa) and np.array_equal(vg, va)
        xg, vg = B.member(1).get_state()
        xa, va = _alone(native, other[0], x2, v2, 1, 3)
        assert np.array_equal(xg, xa) and np.array_equal(vg, va)
