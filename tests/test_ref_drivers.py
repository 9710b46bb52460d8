"""The reference's own drivers, unmodified, on the GPU library against the same drivers on the
reference library.

oracle/Makefile compiles thirteen of the reference's drivers twice:
- against the reference's sources (oracle/_ref/drv_ref_*);
- against the C++ shim, linked to libmpcd_b200.so (oracle/_ref/drv_b200_*).

These are the step validators, the serial and OpenMP benchmark drivers and the single-phase
tools. Every driver runs on the same small case, and every file it writes must agree:
- integer data (cell counts, masks, types) exactly;
- floating-point data within 1e-9 relative (the benchmark drivers run three free steps, over
  which one-ulp thermal-wall draws may propagate);
- printed metrics within 1e-5 relative (six significant digits).

Timing keys and the output-path tags are skipped.
"""
import os
import subprocess

import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state, write_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def _base(c, o):
    return [c + "params.kv", c + "in_x.bin", c + "in_v.bin", c + "in_type.bin", c + "in_r0.bin", o]


DRIVERS = {
    "main_step01_stream_bc_collision": lambda c, o: _base(c, o) + ["1", "1"],
    "main_step02_zone_pass": lambda c, o: _base(c, o) + ["shifted", "1", "1"],
    "main_step03_double_zone_pass": lambda c, o: _base(c, o) + ["1", "1"],
    "main_step04_liquid_closure": lambda c, o: [c + "params.kv", c + "in_x.bin", c + "in_v.bin", c + "red_x.bin",
                                                c + "red_v.bin", c + "in_type.bin", c + "in_r0.bin", o, "1", "1", "1"],
    "main_step05_full_step": lambda c, o: _base(c, o) + ["1", "1"],
    "main_step06_openmp_base_validate": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_step07_openmp_double_validate": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_step08_openmp_full_validate": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_step08_openmp_full_validate_sharedref": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_step09_openmp_full_validate_syncserial": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_benchmark_poiseuille": lambda c, o: _base(c, o) + ["1", "1"],
    "main_benchmark_poiseuille_openmp": lambda c, o: _base(c, o) + ["1", "1", "2"],
    "main_benchmark_poiseuille_openmp_profiled": lambda c, o: _base(c, o) + ["1", "1", "2"],
}


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("drivers"))
    p = poiseuille_params(40, 20, 10)
    x, v = uniform_state(p, 5)
    c = os.path.join(d, "case") + os.sep
    write_case(c, p, x, v, {"benchmark_nSteps": 3, "benchmark_metricsEvery": 1, "benchmark_dumpSteps": "0,3"})
    xr, vr = modulated_state(p, 6)
    xr.tofile(c + "red_x.bin")
    vr.tofile(c + "red_v.bin")
    return p, c, d


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if a.shape != b.shape:
        return np.inf
    if a.size == 0:
        return 0.0
    both_nan = np.isnan(a) & np.isnan(b)
    d = np.where(both_nan, 0.0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))
    return float(np.nanmax(np.where(np.isnan(d), np.inf, d)))


def _compare_bin(path_g, path_r, Nc, name):
    g, r = open(path_g, "rb").read(), open(path_r, "rb").read()
    if g == r:
        return
    assert len(g) == len(r), (name, len(g), len(r))
    if "cellfields" in name:
        assert g[:8] == r[:8], name
        ng, nr = np.frombuffer(g[8:8 + 4 * Nc], np.int32), np.frombuffer(r[8:8 + 4 * Nc], np.int32)
        assert np.array_equal(ng, nr), (name, "N")
        assert _rel(np.frombuffer(g[8 + 4 * Nc:], np.float64), np.frombuffer(r[8 + 4 * Nc:], np.float64)) <= 1e-9, name
    elif name.endswith("_type.bin"):
        raise AssertionError(name)
    elif len(g) == 8 + 4 * Nc:  # int32 grid
        raise AssertionError(name)
    elif len(g) == 8 + 8 * Nc:  # float64 grid
        assert g[:8] == r[:8], name
        assert _rel(np.frombuffer(g[8:], np.float64), np.frombuffer(r[8:], np.float64)) <= 1e-9, name
    else:  # particle arrays
        assert _rel(np.frombuffer(g, np.float64), np.frombuffer(r, np.float64)) <= 1e-9, name


# The closure's optimal beta is num/den summed over all cells. When den falls below the
# reference's own reliability bound (kBetaRepairDenMin = 1e-20, src/liquid_closure.cpp:347),
# the per-cell terms are rounding noise and num sums such terms of both signs: the summation
# order (sequential there, a fixed tree here) decides its value, and the reference itself
# falls back to betaRepair.
BETA_NOISE = ("betaRepairOpt", "betaRepairNum", "finalBetaRepairOpt", "finalBetaRepairNum")


def _beta_unreliable(row):
    den = row.get("betaRepairDen", row.get("finalBetaRepairDen"))
    return den is not None and float(den) < 1e-20


def _skip_key(k):
    kl = k.lower()
    return kl.startswith("time") or kl.startswith("frac") or k in ("inputTag", "outputTag")


def _num_close(a, b):
    try:
        fa, fb = float(a), float(b)
    except ValueError:
        return a == b
    if np.isnan(fa) and np.isnan(fb):
        return True
    return abs(fa - fb) <= 1e-5 * max(abs(fb), 1e-7) + 1e-12


def _compare_text(path_g, path_r, name):
    G = open(path_g).read().splitlines()
    R = open(path_r).read().splitlines()
    if name.endswith(".csv"):
        assert G[0] == R[0] and len(G) == len(R), name
        cols = R[0].split(",")
        for lg, lr in zip(G[1:], R[1:]):
            row = dict(zip(cols, lr.split(",")))
            for k, a, b in zip(cols, lg.split(","), lr.split(",")):
                if _skip_key(k) or k.startswith("nThreads") or (k in BETA_NOISE and _beta_unreliable(row)):
                    continue
                assert _num_close(a, b), (name, k, a, b)
    else:
        kg = dict(l.split("=", 1) for l in G if "=" in l)
        kr = dict(l.split("=", 1) for l in R if "=" in l)
        assert set(kg) == set(kr), (name, set(kg) ^ set(kr))
        for k in kr:
            if _skip_key(k) or k.startswith("nThreads") or (k in BETA_NOISE and _beta_unreliable(kr)):
                continue
            assert _num_close(kg[k], kr[k]), (name, k, kg[k], kr[k])


@pytest.mark.parametrize("driver", sorted(DRIVERS))
def test_reference_driver_on_gpu_library(case, driver):
    p, c, d = case
    exes = {k: os.path.join(REF, f"drv_{k}_{driver}") for k in ("ref", "b200")}
    for e in exes.values():
        if not os.path.exists(e):
            pytest.fail(f"not built: {e} (run __graft_entry__.build() where the reference sources are present)")
    outs = {}
    for k, e in exes.items():
        od = os.path.join(d, driver, k)
        os.makedirs(od, exist_ok=True)
        r = subprocess.run([e] + DRIVERS[driver](c, os.path.join(od, "out")), capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, (k, r.stderr[-400:])
        outs[k] = od
    files = sorted(os.listdir(outs["ref"]))
    assert files == sorted(os.listdir(outs["b200"]))
    assert files, "the driver wrote nothing"
    for f in files:
        pg, pr = os.path.join(outs["b200"], f), os.path.join(outs["ref"], f)
        if f.endswith(".bin"):
            _compare_bin(pg, pr, p["Nc"], f)
        else:
            _compare_text(pg, pr, f)
