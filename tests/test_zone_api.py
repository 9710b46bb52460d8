"""The per-zone API of the reference's include/zone_pass.h on the GPU library against the
reference library.

oracle/zone_api_driver.cpp uses only the reference's headers and calls build_zone_layout,
build_particle_ids_in_zone and run_zone_kernel_inplace. oracle/Makefile compiles it against
the reference's own sources (oracle/_ref/zone_api_ref) and against the C++ shim over
libmpcd_b200.so (oracle/_ref/zone_api_b200). Both run on the same cases and must agree:
  - the layout (zone ids, cell lists, masks, owner map) and the particle-id lists: exactly;
  - the state after each zone's kernel: exactly (positions and velocities);
  - the zone statistics: counts exactly; corrRmsDU, corrMaxDU, occStd, outBand and the rms
    diagnostics within 1e-12 relative. The global momentum and energy changes (diag[2],
    diag[5]) are differences of two sums over all particles, which the GPU adds in another
    order: they agree within 1e-9 absolute.
"""
import os
import subprocess

import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state, write_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

CASES = [
    ("channel_40x30_base", dict(), "uniform", "base", 3),
    ("checker_40x30_shifted", dict(), "checker", "shifted", 4),
    ("odd_tiles_7x9_lff", dict(zoneTileNx=7, zoneTileNy=9, useLocalFluidFractionThresholds=True, lowThrFloor=2.0,
                               highThrFloor=3.0), "sinx", "shifted", 5),
    ("walls_single_full", dict(boundary_left="thermalize", boundary_right="specular", zoneSingleFullDomainMode=True),
     "checker", "single_full", 1),
]


def _run(exe, case_dir, out, mode, seed, stride):
    cmd = [os.path.join(REF, exe), case_dir + "params.kv", case_dir + "in_x.bin", case_dir + "in_v.bin", out, mode,
           str(seed), str(stride)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, exe + ": " + r.stdout + r.stderr


@pytest.mark.parametrize("name,over,kind,mode,stride", CASES, ids=[c[0] for c in CASES])
def test_zone_api_matches_reference(tmp_path, name, over, kind, mode, stride):
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    for exe in ("zone_api_ref", "zone_api_b200"):
        if not os.path.exists(os.path.join(REF, exe)):
            pytest.fail(f"oracle/_ref/{exe} missing (built by oracle/Makefile from the reference sources)")
    p = poiseuille_params(40, 30, 10, **over)
    x, v = uniform_state(p, 11) if kind == "uniform" else modulated_state(p, 11, mode=kind)
    case = str(tmp_path / "case") + os.sep
    write_case(case, p, x, v)
    seed = 88172645463325252
    ro, go = str(tmp_path / "r_"), str(tmp_path / "g_")
    _run("zone_api_ref", case, ro, mode, seed, stride)
    _run("zone_api_b200", case, go, mode, seed, stride)
    lay_r, lay_g = open(ro + "layout.bin", "rb").read(), open(go + "layout.bin", "rb").read()
    assert lay_r == lay_g, "layout"
    nz = int(np.frombuffer(lay_r[:4], np.int32)[0])
    zones = list(range(0, nz, stride))
    assert zones
    moved = 0
    for z in zones:
        pre = f"zone{z}_"
        for part in ("ids", "x", "v"):
            a, b = open(ro + pre + part + ".bin", "rb").read(), open(go + pre + part + ".bin", "rb").read()
            assert a == b, (z, part)
        sr = np.fromfile(ro + pre + "stats.bin")
        sg = np.fromfile(go + pre + "stats.bin")
        assert sr.shape == sg.shape == (18,)
        exact = [0, 1, 2, 3, 16, 17]  # nHigh, nLow, moved out, moved in, movedDense, movedSparse
        assert np.array_equal(sr[exact], sg[exact]), (z, sr[exact], sg[exact])
        rel = [4, 5, 6, 7, 9, 10, 14, 15]  # corrRmsDU, corrMaxDU, occStd, outBand, rms dPx, rms dPy, rms ux, rms uy
        d = np.abs(sr[rel] - sg[rel]) / np.maximum(1.0, np.abs(sr[rel]))
        assert d.max() <= 1e-12, (z, sr[rel], sg[rel])
        for k in (8, 11):  # |dP global|, dE
            assert abs(sr[k] - sg[k]) <= 1e-9, (z, k, sr[k], sg[k])
        assert np.isnan(sr[12]) and np.isnan(sg[12]) and sr[13] == sg[13] == 0.0
        moved += int(sr[16] + sr[17])
    assert moved > 0  # the case moves particles
