"""The oracle (oracle/mpcd_oracle.c) pinned against the reference.

1. RNG known-answer vectors produced by libstdc++ itself (tests/golden/rng_kat.cpp).
2. Golden fixtures produced by the unmodified reference (tests/golden/make_golden.py):
   every phase of one benchmark step must be bit-identical.
3. Where the reference library is built (oracle/_ref), a sweep of parameter variants run
   through both, bit-identical.
"""
import ctypes as C
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state
from tests.golden.make_golden import STEP, build_params, make_state

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kat_lines():
    with open(os.path.join(GOLD, "rng_kat.txt")) as f:
        return [ln.split() for ln in f]


def test_rng_kat(oracle):
    L = oracle.lib
    L.oracle_rng_kat.argtypes = [C.c_uint64, C.c_int, C.c_int, np.ctypeslib.ndpointer(np.float64), np.ctypeslib.ndpointer(np.uint64)]
    L.oracle_shuffle_kat.argtypes = [C.c_uint64, C.c_int, np.ctypeslib.ndpointer(np.int32)]
    kinds = {"raw": 0, "u01": 1, "normal": 2, "ubin": 3, "uint": 4}
    checked = 0
    for tok in _kat_lines():
        if tok[0] == "shuffle":
            seed, n = int(tok[1]), int(tok[2])
            a = np.arange(n, dtype=np.int32)
            L.oracle_shuffle_kat(seed, n, a)
            assert a.tolist() == [int(t) for t in tok[3:]], (seed, n)
        else:
            seed = int(tok[1])
            vals = tok[2:]
            d = np.zeros(len(vals))
            u = np.zeros(len(vals), np.uint64)
            L.oracle_rng_kat(seed, kinds[tok[0]], len(vals), d, u)
            if tok[0] in ("u01", "normal"):
                assert np.array_equal(d, np.array([float.fromhex(t) for t in vals])), tok[0]
            else:
                assert u.tolist() == [int(t) for t in vals], tok[0]
        checked += 1
    assert checked >= 50


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _run_oracle_case(O, p, x, v):
    s = STEP
    out = {"in_x": x, "in_v": v}
    x1, v1 = O.stream(p, x, v)
    x1, v1, wall = O.apply_bc(p, x1, v1, 104729 + 10007 * s)
    out["bc_x"], out["bc_v"] = x1, v1
    cid = O.srd_shift_cells(p, x1, 130363 + 10007 * s)
    out["srd_cid"] = cid
    v2 = O.srd_collide(p, v1, cid, 433494437 + 10007 * s)
    out["coll_v"] = v2
    rho_t = p["gamma"] / ((p["Lx"] / p["Nx"]) * (p["Ly"] / p["Ny"]))
    f = O.cell_fields(p, x1, v2, rho_t)
    for k in ("N", "Px", "Py", "T", "P"):
        out["fields_" + k] = f[k]
    xb, vb, mb = O.zone_pass(p, x1, v2, "base", 88172645463325252 + 10007 * s)
    out["base_x"], out["base_v"] = xb, vb
    xs, vs, ms = O.zone_pass(p, xb, vb, "shifted", 88172645463325252 + 4099 + 10007 * s)
    out["shifted_x"], out["shifted_v"] = xs, vs
    xo, vo, mc, det = O.liquid_closure(p, x1, v2, xs, vs)
    out["closure_x"], out["closure_v"] = xo, vo
    for k in ("pdrive", "duRepairX", "duEOSX", "interzoneMask"):
        out["closure_" + k] = det[k]
    xf, vf, _ = O.step(p, x, v, s)
    out["step_x"], out["step_v"] = xf, vf
    return out, wall, mb, ms, mc


@pytest.mark.parametrize("case", sorted(os.path.basename(f)[:-5] for f in glob.glob(os.path.join(GOLD, "*.json"))))
def test_golden_case(oracle, case):
    meta = json.load(open(os.path.join(GOLD, case + ".json")))
    from tests.golden.make_golden import CASES
    over, kind, seed, keep = CASES[case]
    p = build_params(over)
    z = np.load(os.path.join(GOLD, case + ".npz"))
    out, wall, mb, ms, mc = _run_oracle_case(oracle, p, z["in_x"], z["in_v"])
    for k, dig in meta["digests"].items():
        if keep:
            assert np.array_equal(out[k], z[k]), k
        assert _digest(out[k]) == dig, k
    assert wall == meta["wall"]
    assert [mb["nParticlesMovedDense"], mb["nParticlesMovedSparse"]] == meta["base_moved"]
    assert [ms["nParticlesMovedDense"], ms["nParticlesMovedSparse"]] == meta["shifted_moved"]
    for k, val in meta["closure"].items():
        assert mc[k] == val, k


VARIANTS = [
    ("default_40x30", dict(), "uniform"),
    ("odd_tiles", dict(zoneTileNx=7, zoneTileNy=9), "checker"),
    ("tile_not_dividing", dict(zoneTileNx=6, zoneTileNy=4), "siny"),
    ("no_thermostat_keepmean", dict(useThermostat=False, keepMeanFlow=True), "uniform"),
    ("no_momcorr", dict(enableMomentumCorrectionPostRedistribution=False), "sinx"),
    ("lff_thresholds", dict(useLocalFluidFractionThresholds=True, lowThrFloor=2.0, highThrFloor=3.0), "checker"),
    ("override_low", dict(lowThrBulkOverride=8.5, highMode="1+coef"), "sinx"),
    ("walls_all", dict(boundary_left="thermalize", boundary_right="specular", boundary_bottom="bounceback",
                       boundary_top="thermalize", Utop=0.5, Ubottom=-0.2), "uniform"),
    ("periodic_y", dict(boundary_bottom="periodic", boundary_top="periodic", g=0.01), "siny"),
    ("no_closure_smoothing", dict(smoothPdriveAtInterzone=False, betaRepair=0.3, useOptimalBetaRepair=False), "uniform"),
    ("passthrough", dict(zonePassthroughMode=True, smoothPdriveInterzoneWidthCells=0, smoothPdriveInterzoneBlend=0.5), "checker"),
    ("three_passes_ppc5", dict(maxRedistribPasses=3, gamma=5.0), "checker"),
]


@pytest.mark.parametrize("name,over,kind", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_oracle_matches_reference(oracle, reference, name, over, kind):
    ppc = 5 if "ppc5" in name else 10
    p = poiseuille_params(40, 30, ppc, **over)
    x, v = uniform_state(p, 5) if kind == "uniform" else modulated_state(p, 5, mode=kind)
    out_o = _run_oracle_case(oracle, p, x, v)[0]
    out_r = _run_oracle_case(reference, p, x, v)[0]
    for k in out_o:
        assert np.array_equal(out_o[k], out_r[k]), k


def test_oracle_multistep_matches_reference(oracle, reference):
    p = poiseuille_params(30, 30, 10)
    x, v = uniform_state(p, 9)
    xo, vo, xr, vr = x, v, x, v
    for s in range(1, 6):
        xo, vo, mo = oracle.step(p, xo, vo, s)
        xr, vr, mr = reference.step(p, xr, vr, s)
        assert np.array_equal(xo, xr) and np.array_equal(vo, vr), s
        for k in ("occStd", "outBand", "meanKinetic", "meanUx", "Qx", "baseOccStd", "shiftedOutBand"):
            assert mo[k] == mr[k], (s, k)


SERIAL_VARIANTS = ["default_40x30", "odd_tiles", "tile_not_dividing", "walls_all", "periodic_y", "lff_thresholds"]


@pytest.mark.parametrize("name", SERIAL_VARIANTS)
def test_oracle_serial_pass_matches_reference(oracle, reference, name):
    """run_zone_pass (zones in sequence, in place): oracle restatement vs the reference."""
    over, kind = {v[0]: (v[1], v[2]) for v in VARIANTS}[name]
    p = poiseuille_params(40, 30, 10, **over)
    x, v = uniform_state(p, 7) if kind == "uniform" else modulated_state(p, 7, mode=kind)
    for mode, seed in (("base", 88172645463325252), ("shifted", 998244353)):
        xo, vo, mo = oracle.zone_pass_serial(p, x, v, mode, seed)
        xr, vr, mr = reference.zone_pass_serial(p, x, v, mode, seed)
        assert np.array_equal(xo, xr) and np.array_equal(vo, vr), mode
        for k in ("nZones", "nParticlesMovedDense", "nParticlesMovedSparse", "corrRmsDU", "corrMaxDU"):
            assert mo[k] == mr[k], (mode, k)
        x, v = xo, vo
