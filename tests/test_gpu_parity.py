"""CUDA path vs the oracle, phase by phase, through the C-ABI (libmpcd_b200.so).

Bar (the reference's contract for the plain FP64 form):
  - cell ids, counts, zone ownership and moved-particle sets: bit-exact;
  - positions: bit-exact (they never depend on quantities computed in a different order);
  - velocities: within 1e-12 relative per step. The only sources of non-bit-exactness are
    (a) glibc's log, which the thermal-wall Gaussian draws use and which is not correctly
        rounded in ~0.08% of inputs (the device uses a correctly rounded log: those draws
        differ by one ulp), and
    (b) the liquid closure's global beta_opt numerator/denominator, summed in a fixed tree
        order instead of the reference's sequential cell order.
"""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state
from tests.parity_checks import check_phases

pytestmark = pytest.mark.gpu

REL = 1e-12
S = 3  # step number of the seed schedule


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def vclose(a, b, rel=REL):
    d = np.abs(a - b) / np.maximum(1.0, np.abs(b))
    return float(d.max()) if d.size else 0.0


CASES = [
    ("channel_40x30", dict(Nx=40, Ny=30, ppc=10), "uniform", 21),
    ("modulated_30x20_tiles7x6", dict(Nx=30, Ny=20, ppc=10, zoneTileNx=7, zoneTileNy=6), "sinx", 22),
    ("checker_32x24_ppc12", dict(Nx=32, Ny=24, ppc=12), "checker", 23),
    ("walls_24x16_lff", dict(Nx=24, Ny=16, ppc=12, boundary_left="bounceback", boundary_right="bounceback",
                             boundary_bottom="specular", boundary_top="thermalize", Utop=0.3,
                             useLocalFluidFractionThresholds=True, highMode="1+coef", lowMode="1+coef",
                             lowThrFloor=3.0, highThrFloor=4.0), "checker", 24),
    ("single_full_16x12", dict(Nx=16, Ny=12, ppc=10, zoneSingleFullDomainMode=True), "uniform", 25),
    ("periodic_y_g", dict(Nx=20, Ny=20, ppc=10, boundary_bottom="periodic", boundary_top="periodic", g=0.01), "siny", 26),
]


def make_case(over, kind, seed):
    over = dict(over)
    Nx, Ny, ppc = over.pop("Nx"), over.pop("Ny"), over.pop("ppc")
    p = poiseuille_params(Nx, Ny, ppc, **over)
    x, v = uniform_state(p, seed) if kind == "uniform" else modulated_state(p, seed, mode=kind)
    return p, x, v


@pytest.mark.parametrize("name,over,kind,seed", CASES, ids=[c[0] for c in CASES])
def test_phases_match_oracle(oracle, name, over, kind, seed):
    native = _native()
    p, x, v = make_case(over, kind, seed)
    check_phases(native, oracle, p, x, v, S)


@pytest.mark.parametrize("name,over,kind,seed", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_step_matches_oracle(oracle, name, over, kind, seed):
    native = _native()
    p, x, v = make_case(over, kind, seed)
    with native.Context(p) as ctx:
        xo, vo = x, v
        for s in range(1, 4):
            ctx.set_state(xo, vo)  # identical input every step (the per-step contract)
            m = ctx.step(s - 1, 1, metrics=True)
            xg, vg = ctx.get_state()
            xo, vo, mo = oracle.step(p, xo, vo, s)
            assert np.array_equal(xg, xo), f"step {s} positions"
            assert vclose(vg, vo) <= REL, f"step {s} velocities"
            assert m["base"]["nParticlesMovedDense"] == mo["base"]["nParticlesMovedDense"]
            assert m["shifted"]["nParticlesMovedSparse"] == mo["shifted"]["nParticlesMovedSparse"]
            for k in ("occStd", "outBand", "baseOccStd", "shiftedOutBand", "meanKinetic", "meanUx", "Qx"):
                assert abs(m[k] - mo[k]) <= 1e-10 * max(1.0, abs(mo[k])), (s, k, m[k], mo[k])


def test_free_run_tracks_oracle(oracle):
    native = _native()
    p, x, v = make_case(dict(Nx=30, Ny=30, ppc=10), "uniform", 31)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        ctx.step(0, 4)
        xg, vg = ctx.get_state()
    xo, vo = x, v
    for s in range(1, 5):
        xo, vo, _ = oracle.step(p, xo, vo, s)
    # no teacher forcing: one-ulp differences of thermal draws may propagate, nothing more
    assert vclose(xg, xo) <= 1e-9
    assert vclose(vg, vo) <= 1e-9


def test_golden_fixtures_on_gpu():
    """The reference's own outputs (tests/golden) reproduced by the CUDA path."""
    import json
    import os
    native = _native()
    from tests.golden.make_golden import CASES as GC, build_params
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for name, (over, kind, seed, keep) in GC.items():
        if not keep:
            continue
        p = build_params(over)
        z = np.load(os.path.join(gold, name + ".npz"))
        with native.Context(p) as ctx:
            ctx.set_state(z["bc_x"], z["bc_v"])
            ctx.srd_collide_cells(z["srd_cid"], 433494437 + 10007 * S)
            _, vg = ctx.get_state()
            assert np.array_equal(vg, z["coll_v"]), name
            ctx.save_ref()
            ctx.zone_pass("base", 88172645463325252 + 10007 * S)
            xg, vg = ctx.get_state()
            assert np.array_equal(xg, z["base_x"]) and np.array_equal(vg, z["base_v"]), name
            ctx.zone_pass("shifted", 88172645463325252 + 4099 + 10007 * S)
            xg, vg = ctx.get_state()
            assert np.array_equal(xg, z["shifted_x"]) and np.array_equal(vg, z["shifted_v"]), name
            ctx.liquid_closure()
            xg, vg = ctx.get_state()
            assert np.array_equal(xg, z["closure_x"]) and vclose(vg, z["closure_v"]) <= REL, name
            ctx.set_state(z["in_x"], z["in_v"])
            ctx.step(S - 1, 1)
            xg, vg = ctx.get_state()
            assert np.array_equal(xg, z["step_x"]) and vclose(vg, z["step_v"]) <= REL, name
