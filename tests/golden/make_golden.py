"""Generates tests/golden/*.npz from the UNMODIFIED reference (oracle/_ref/libmpcdref.so,
built by oracle/Makefile from the reference's own sources).

Each case runs the reference's phases in the order of one benchmark step
(src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:241-279) with the
benchmark's seed schedule, and records every intermediate. Small cases keep the arrays;
larger ones keep SHA-256 digests of the raw little-endian bytes.

Run from the repository root:  python -m tests.golden.make_golden
"""
import hashlib
import json
import os

import numpy as np

from src_incompressible_openmp_b200.cases import modulated_state, poiseuille_params, uniform_state
from tests.oracle_libs import Reference

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (params overrides, state kind, seed, keep arrays)
    "channel_20x10": (dict(Nx=20, Ny=10, ppc=10), "uniform", 11, True),
    "single_full_16x12": (dict(Nx=16, Ny=12, ppc=10, zoneSingleFullDomainMode=True), "uniform", 14, True),
    "modulated_30x20_tiles7x6": (dict(Nx=30, Ny=20, ppc=10, zoneTileNx=7, zoneTileNy=6), "sinx", 12, False),
    "walls_24x16_lff": (
        dict(Nx=24, Ny=16, ppc=12, boundary_left="bounceback", boundary_right="bounceback", boundary_bottom="specular",
             boundary_top="thermalize", Utop=0.3, useLocalFluidFractionThresholds=True, highMode="1+coef",
             lowMode="1+coef", lowThrFloor=3.0, highThrFloor=4.0),
        "checker", 13, False),
}

STEP = 3


def build_params(over):
    over = dict(over)
    Nx, Ny, ppc = over.pop("Nx"), over.pop("Ny"), over.pop("ppc")
    return poiseuille_params(Nx, Ny, ppc, **over)


def make_state(p, kind, seed):
    if kind == "uniform":
        return uniform_state(p, seed)
    return modulated_state(p, seed, mode=kind)


def run_case(R, p, x, v):
    s = STEP
    out = {"in_x": x, "in_v": v}
    x1, v1 = R.stream(p, x, v)
    x1, v1, wall = R.apply_bc(p, x1, v1, 104729 + 10007 * s)
    out["bc_x"], out["bc_v"] = x1, v1
    cid = R.srd_shift_cells(p, x1, 130363 + 10007 * s)
    out["srd_cid"] = cid
    v2 = R.srd_collide(p, v1, cid, 433494437 + 10007 * s)
    out["coll_v"] = v2
    rho_t = p["gamma"] / ((p["Lx"] / p["Nx"]) * (p["Ly"] / p["Ny"]))
    f = R.cell_fields(p, x1, v2, rho_t)
    for k in ("N", "Px", "Py", "T", "P"):
        out["fields_" + k] = f[k]
    xb, vb, mb = R.zone_pass(p, x1, v2, "base", 88172645463325252 + 10007 * s)
    out["base_x"], out["base_v"] = xb, vb
    xs, vs, ms = R.zone_pass(p, xb, vb, "shifted", 88172645463325252 + 4099 + 10007 * s)
    out["shifted_x"], out["shifted_v"] = xs, vs
    xo, vo, mc, det = R.liquid_closure(p, x1, v2, xs, vs)
    out["closure_x"], out["closure_v"] = xo, vo
    for k in ("pdrive", "duRepairX", "duEOSX", "interzoneMask"):
        out["closure_" + k] = det[k]
    xf, vf, mstep = R.step(p, x, v, s)
    out["step_x"], out["step_v"] = xf, vf
    meta = {
        "wall": wall,
        "base_moved": [mb["nParticlesMovedDense"], mb["nParticlesMovedSparse"]],
        "shifted_moved": [ms["nParticlesMovedDense"], ms["nParticlesMovedSparse"]],
        "closure": {k: mc[k] for k in ("betaRepairOpt", "betaRepairApplied", "betaRepairNum", "betaRepairDen",
                                       "meanPdriveRaw", "meanPdrive", "nMaskedInterzoneCells")},
        "step_occStd": mstep["occStd"], "step_meanKinetic": mstep["meanKinetic"], "step_Qx": mstep["Qx"],
    }
    return out, meta


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    R = Reference()
    for name, (over, kind, seed, keep) in CASES.items():
        p = build_params(over)
        x, v = make_state(p, kind, seed)
        arrays, meta = run_case(R, p, x, v)
        meta["params"] = {k: (None if isinstance(val, float) and val != val else val) for k, val in p.items()}
        meta["state"] = [kind, seed]
        meta["digests"] = {k: digest(a) for k, a in arrays.items()}
        if keep:
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        else:
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), in_x=arrays["in_x"], in_v=arrays["in_v"])
        with open(os.path.join(HERE, f"{name}.json"), "w") as fh:
            json.dump(meta, fh, indent=1, sort_keys=True)
        print(name, "n =", p["n"], "moved", meta["base_moved"], meta["shifted_moved"])


if __name__ == "__main__":
    main()
