"""Batched replicas of the fast form (mpcd_batch_create_form with MPCD_FORM_FAST): every phase of
a step is one launch for all replicas, and each replica's state is bit-identical to the same
replica stepped alone, across calls, odd step counts (the bins' orientation flips), a member
stepped on its own in between, and the collision's spill path."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import ensemble_family, modulated_state, poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu

REPLICAS = [
    (dict(Nx=40, Ny=20, ppc=10), "uniform", 61),
    (dict(Nx=24, Ny=16, ppc=8, bodyForceX=3e-3), "uniform", 62),
    (dict(Nx=30, Ny=30, ppc=12, bodyForceX=2e-4), "sinx", 63),
    (dict(Nx=64, Ny=18, ppc=20, bodyForceX=1e-2), "uniform", 64),
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


# the schedule: (who, step0, nsteps); who "batch" steps every replica together, an int steps
# that replica alone
SCHEDULE = [("batch", 0, 7), ("batch", 7, 4), (0, 11, 1), ("batch", 12, 3)]


def _alone(native, cases):
    out = []
    for i, (p, x, v) in enumerate(cases):
        with native.Context(p, form="fast") as c:
            c.set_state(x, v)
            for who, s0, k in SCHEDULE:
                if who == "batch" or who == i:
                    c.step(s0, k)
            out.append(c.get_state())
    return out


def _batched(native, cases):
    B = native.Batch([p for p, _, _ in cases], form="fast")
    try:
        for i, (p, x, v) in enumerate(cases):
            B.member(i).set_state(x, v)
        for who, s0, k in SCHEDULE:
            if who == "batch":
                t = B.step(s0, k)
                assert t > 0.0
            else:
                B.member(who).step(s0, k)
        return [B.member(i).get_state() for i in range(len(cases))]
    finally:
        B.close()


def _compare(got, want):
    for i, ((xb, vb), (xa, va)) in enumerate(zip(got, want)):
        assert np.all(np.isfinite(xb)) and np.all(np.isfinite(vb)), i
        assert np.array_equal(xb, xa), i
        assert np.array_equal(vb, va), i


def test_fast_batch_equals_replicas_alone():
    native = _native()
    cases = [_case(*r) for r in REPLICAS]
    _compare(_batched(native, cases), _alone(native, cases))


def test_fast_batch_graph_replay_equals_eager(monkeypatch):
    # batched steps replayed from CUDA graphs (the default) against the same steps launched
    # one kernel at a time
    native = _native()
    cases = [_case(*r) for r in REPLICAS]
    replayed = _batched(native, cases)
    monkeypatch.setenv("MPCD_FAST_BATCH_GRAPHS", "0")
    _compare(_batched(native, cases), replayed)


def test_fast_batch_spill_path(monkeypatch):
    # a small staging capacity sends fuller collision tiles to the spill kernel, in the batch
    # as in the replicas alone
    native = _native()
    monkeypatch.setenv("MPCD_FAST_COLLIDE_PCAP", "64")
    cases = [_case(*r) for r in REPLICAS[2:]]
    _compare(_batched(native, cases), _alone(native, cases))


def test_fast_batch_ensemble_family_conserves_mass():
    # a slice of the benchmark's ensemble family: every particle kept, momentum finite
    native = _native()
    reps = ensemble_family(12, 2024)
    B = native.Batch([p for p, _ in reps], form="fast")
    try:
        for i, (p, seed) in enumerate(reps):
            x, v = uniform_state(p, seed)
            B.member(i).set_state(x, v)
        B.step(0, 20)
        for i, (p, _) in enumerate(reps):
            x, v = B.member(i).get_state()
            assert x.shape[0] == 2 * p["n"]
            assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
            assert np.all((x[0::2] >= 0) & (x[0::2] < p["Lx"]) & (x[1::2] >= 0) & (x[1::2] <= p["Ly"]))
    finally:
        B.close()


def test_fast_batch_rejects_learned_members():
    native = _native()
    cases = [_case(*r) for r in REPLICAS[:2]]
    B = native.Batch([p for p, _, _ in cases], form="fast")
    try:
        for i, (p, x, v) in enumerate(cases):
            B.member(i).set_state(x, v)
        net = native.learned_init(3)
        net[-1] = 1e-3  # the output scale (set by training otherwise)
        B.member(1).learned_set(net, 0.0)
        with pytest.raises(native.MpcdError):
            B.step(0, 1)
    finally:
        B.close()
