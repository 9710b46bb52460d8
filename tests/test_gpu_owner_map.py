"""mpcd_zone_owner_map (the zone layouts' owner grids, src/zone_pass.cpp:160-221,1049-1063) against
the oracle and, where it is built, the compiled reference, for the base, shifted and single
full-domain layouts on even, ragged and non-periodic grids."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params

pytestmark = pytest.mark.gpu

GRIDS = [
    dict(Nx=50, Ny=50),
    dict(Nx=37, Ny=23),
    dict(Nx=64, Ny=40, zoneTileNx=8, zoneTileNy=12),
    dict(Nx=30, Ny=20, boundary_left="bounceback", boundary_right="bounceback"),
]


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def _params(g):
    g = dict(g)
    Nx, Ny = g.pop("Nx"), g.pop("Ny")
    return poiseuille_params(Nx, Ny, 5, **g)


@pytest.mark.parametrize("mode", ["base", "shifted", "single_full"])
@pytest.mark.parametrize("g", GRIDS, ids=[f"{g['Nx']}x{g['Ny']}" for g in GRIDS])
def test_owner_map_matches_oracle(oracle, g, mode):
    native = _native()
    p = _params(g)
    with native.Context(p) as c:
        got = c.zone_owner_map(mode)
    want = oracle.zone_owner_map(p, mode)
    assert got.shape == (p["Nc"],)
    assert np.all(got >= 0)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("mode", ["base", "shifted"])
def test_owner_map_matches_reference(reference, mode):
    native = _native()
    p = _params(GRIDS[1])
    with native.Context(p) as c:
        got = c.zone_owner_map(mode)
    assert np.array_equal(got, reference.zone_owner_map(p, mode))
