"""run_zone_pass (zones one after another, in place) on the GPU against the oracle, which
test_oracle pins to the reference: positions, velocities and metrics bit-exact."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu

CASES = [
    ("channel_40x30", dict(), "uniform"),
    ("odd_tiles_7x9", dict(zoneTileNx=7, zoneTileNy=9), "checker"),
    ("walls_all", dict(boundary_left="thermalize", boundary_right="specular", boundary_bottom="bounceback",
                       boundary_top="thermalize", Utop=0.5, Ubottom=-0.2), "uniform"),
    ("lff", dict(useLocalFluidFractionThresholds=True, lowThrFloor=2.0, highThrFloor=3.0), "sinx"),
]


@pytest.mark.parametrize("name,over,kind", CASES, ids=[c[0] for c in CASES])
def test_serial_pass_matches_oracle(oracle, name, over, kind):
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    p = poiseuille_params(40, 30, 10, **over)
    x, v = uniform_state(p, 8) if kind == "uniform" else modulated_state(p, 8, mode=kind)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        xo, vo = x, v
        for mode, seed in (("base", 88172645463325252), ("shifted", 998244353)):
            mg = ctx.zone_pass_serial(mode, seed)
            xg, vg = ctx.get_state()
            xo, vo, mo = oracle.zone_pass_serial(p, xo, vo, mode, seed)
            assert np.array_equal(xg, xo), f"{mode} positions"
            assert np.array_equal(vg, vo), f"{mode} velocities"
            for k in ("nZones", "nParticlesMovedDense", "nParticlesMovedSparse", "corrMaxDU"):
                assert mg[k] == mo[k], (mode, k)
            assert abs(mg["corrRmsDU"] - mo["corrRmsDU"]) <= 1e-12 * max(1.0, mo["corrRmsDU"])
