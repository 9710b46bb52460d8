"""Parameters, named workloads, synthetic states and the reference's file formats.

- ``poiseuille_params(Nx, Ny, ppc, ...)`` builds the parameter set of the Poiseuille channel
  benchmark with the reference's key names (include/types.h:10-72); defaults follow the
  reference's MATLAB case builder (matlab/build_benchmark_poiseuille_params_equal.m:30-85)
  with the channel workload's physics: a = 0.2, dt = 0.1, alpha = 130 deg (radians in the
  file), body force 1e-3 along +x, periodic x, thermalising walls at y = 0 and y = Ly,
  10x10 tiles with a shifted second pass, Kvirial 1.
- ``uniform_state(params, seed)`` draws the seeded synthetic initial state the reference's
  case builder describes (matlab/build_ad_hoc_state_uniform.m:27-40): positions uniform in
  the box, Maxwellian velocities with variance kBT and the mean removed. numpy's
  default_rng stands in for MATLAB's generator; the .bin contents are the contract.
- ``write_params_kv`` / ``read_params_kv`` and the .bin helpers follow the reference's
  formats (src/params_io.cpp:21-137, src/state_io.cpp:10-68, src/dump_io.cpp:19-39).
"""
import math
import os

import numpy as np

from . import _abi

BOOL_KEYS = (
    "useThermostat", "keepMeanFlow", "noSurfaceCase", "redistributionEnableSurfaceTopology",
    "redistributionWallWettingEnabled", "useInterfaceVelocityReorientation", "useIncompressibleRedistribution",
    "redistribAfterCollision", "useZoneRedistribution", "zoneUseShiftedSecondPass", "zonePassthroughMode",
    "zoneSingleFullDomainMode", "enableMomentumCorrectionPostRedistribution", "useLocalFluidFractionThresholds",
    "useLiquidClosure", "useOptimalBetaRepair", "smoothPdriveAtInterzone", "smoothPdriveIncludeShiftedLayouts",
)
INT_KEYS = ("Nx", "Ny", "Nc", "n", "zoneTileNx", "zoneTileNy", "maxRedistribPasses", "smoothPdriveInterzoneWidthCells")
STR_KEYS = ("boundary_left", "boundary_right", "boundary_bottom", "boundary_top", "highMode", "lowMode")
FLOAT_KEYS = (
    "Lx", "Ly", "dt", "a0", "alpha", "kBT", "g", "bodyForceX", "Utop", "Ubottom", "wallSigma", "gamma", "coef",
    "fluidFracGain", "lowThrFloor", "highThrFloor", "lowThrBulkOverride", "betaRepair", "betaEOS", "Kvirial",
    "smoothPdriveInterzoneBlend",
)
ALL_KEYS = INT_KEYS + FLOAT_KEYS + BOOL_KEYS + STR_KEYS


def poiseuille_params(Nx=50, Ny=50, ppc=10, a=0.2, **over):
    """Parameter dict (reference key names) of the Poiseuille channel on Nx x Ny cells."""
    p = dict(
        Nx=Nx, Ny=Ny, Nc=Nx * Ny, n=int(round(ppc * Nx * Ny)),
        Lx=Nx * a, Ly=Ny * a, dt=0.1, a0=a,
        alpha=130.0 * math.pi / 180.0, kBT=1.0, g=0.0, bodyForceX=1e-3,
        useThermostat=True, keepMeanFlow=False,
        boundary_left="periodic", boundary_right="periodic", boundary_bottom="thermalize", boundary_top="thermalize",
        Utop=0.0, Ubottom=0.0, wallSigma=1.0,
        noSurfaceCase=True, redistributionEnableSurfaceTopology=False, redistributionWallWettingEnabled=False,
        useInterfaceVelocityReorientation=False, useIncompressibleRedistribution=True, redistribAfterCollision=True,
        useZoneRedistribution=True, zoneTileNx=10, zoneTileNy=10, zoneUseShiftedSecondPass=True,
        zonePassthroughMode=False, zoneSingleFullDomainMode=False, enableMomentumCorrectionPostRedistribution=True,
        gamma=float(ppc), coef=0.1, highMode="coef", lowMode="coef", maxRedistribPasses=2,
        useLocalFluidFractionThresholds=False, fluidFracGain=0.8, lowThrFloor=20.0, highThrFloor=25.0,
        lowThrBulkOverride=float("nan"),
        useLiquidClosure=True, useOptimalBetaRepair=True, betaRepair=0.0, betaEOS=1.0, Kvirial=1.0,
        smoothPdriveAtInterzone=True, smoothPdriveInterzoneWidthCells=2, smoothPdriveInterzoneBlend=1.0,
        smoothPdriveIncludeShiftedLayouts=True,
    )
    p.update(over)
    if "Nc" not in over:
        p["Nc"] = p["Nx"] * p["Ny"]
    return p


# Named workloads: the reference's CPU-runnable channel and the large single-GPU channel.
WORKLOADS = {
    "poiseuille_50x50_ppc10": dict(Nx=50, Ny=50, ppc=10, steps=1500),
    "channel_2048x512_ppc10": dict(Nx=2048, Ny=512, ppc=10, steps=1000),
    "channel_4096x1024_ppc20": dict(Nx=4096, Ny=1024, ppc=20, steps=2000),
}


def ensemble_family(count, seed):
    """Independent Poiseuille channels of uneven size, density and forcing, seeded: Nx uniform in
    [32, 512], Ny in [16, 128], particles per cell in [5, 20], bodyForceX log-uniform in
    [1e-4, 1e-2]; replica r's initial state seed is 1000 + r. Returns [(params, state_seed)]."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        Nx = int(rng.integers(32, 513))
        Ny = int(rng.integers(16, 129))
        ppc = int(rng.integers(5, 21))
        force = float(10.0 ** rng.uniform(-4.0, -2.0))
        out.append((poiseuille_params(Nx, Ny, ppc, bodyForceX=force), 1000 + r))
    return out


def to_c(p):
    """Parameter dict -> include/mpcd_c.h mpcd_params_c."""
    c = _abi.ParamsC()
    for k in INT_KEYS:
        setattr(c, k, int(p[k]))
    for k in FLOAT_KEYS:
        setattr(c, k, float(p[k]))
    for k in BOOL_KEYS:
        setattr(c, k, 1 if p[k] else 0)
    for k in ("boundary_left", "boundary_right", "boundary_bottom", "boundary_top"):
        setattr(c, k, _abi.BC_MODES.get(p[k], _abi.BC_UNKNOWN))
    c.highMode = 1 if p["highMode"] == "1+coef" else 0
    c.lowMode = 1 if p["lowMode"] == "1+coef" else 0
    return c


def uniform_state(p, seed=1):
    """Seeded uniform positions and zero-mean Maxwellian velocities, interleaved (2n,)."""
    rng = np.random.default_rng(seed)
    n = int(p["n"])
    x = np.empty((n, 2))
    x[:, 0] = p["Lx"] * rng.random(n)
    x[:, 1] = p["Ly"] * rng.random(n)
    v = math.sqrt(p["kBT"]) * rng.standard_normal((n, 2))
    v -= v.mean(axis=0)
    return x.reshape(-1).copy(), v.reshape(-1).copy()


def modulated_state(p, seed=1, amp=0.6, mode="sinx"):
    """Positions with a smooth density modulation (forces dense and sparse cells), as the
    reference's matlab/build_ad_hoc_state_modulated.m describes; accept-reject sampling."""
    rng = np.random.default_rng(seed)
    n = int(p["n"])
    out = np.empty((0, 2))
    while out.shape[0] < n:
        cand = rng.random((2 * n, 2)) * np.array([p["Lx"], p["Ly"]])
        if mode == "sinx":
            w = 1.0 + amp * np.sin(2 * np.pi * cand[:, 0] / p["Lx"])
        elif mode == "siny":
            w = 1.0 + amp * np.sin(2 * np.pi * cand[:, 1] / p["Ly"])
        else:
            w = 1.0 + amp * np.sign(np.sin(4 * np.pi * cand[:, 0] / p["Lx"]) * np.sin(4 * np.pi * cand[:, 1] / p["Ly"]))
        keep = rng.random(2 * n) * (1.0 + amp) < w
        out = np.concatenate([out, cand[keep]])
    x = out[:n]
    v = math.sqrt(p["kBT"]) * rng.standard_normal((n, 2))
    v -= v.mean(axis=0)
    return x.reshape(-1).copy(), v.reshape(-1).copy()


def _fmt(v):
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        if math.isnan(v):
            return "NaN"
        return repr(v)
    return str(v)


def write_params_kv(p, path, extra=None):
    """key=value text (matlab/write_params_kv.m:9-24 writes %.17g and true/false)."""
    with open(path, "w") as f:
        for k in ALL_KEYS:
            f.write(f"{k}={_fmt(p[k])}\n")
        for k, v in (extra or {}).items():
            f.write(f"{k}={_fmt(v)}\n")


def read_params_kv(path):
    """Strict reader with the reference's rules (src/params_io.cpp:21-137)."""
    kv = {}
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            if "=" not in line:
                raise ValueError(f"Invalid key=value line in params file: {line}")
            k, v = line.split("=", 1)
            kv[k.strip()] = v.strip()
    p = {}
    for k in ALL_KEYS:
        if k not in kv:
            raise ValueError(f"Missing required params key: {k}")
        s = kv[k]
        if k in INT_KEYS:
            p[k] = int(s)
        elif k in FLOAT_KEYS:
            p[k] = float(s)
        elif k in BOOL_KEYS:
            if s in ("true", "1"):
                p[k] = True
            elif s in ("false", "0"):
                p[k] = False
            else:
                raise ValueError(f"Invalid boolean value: {s}")
        else:
            p[k] = s
    return p, kv


def write_bin(path, arr, dtype=np.float64):
    np.ascontiguousarray(arr, dtype=dtype).tofile(path)


def read_bin(path, count, dtype=np.float64):
    a = np.fromfile(path, dtype=dtype, count=count)
    if a.size != count:
        raise ValueError(f"Cannot read expected payload from: {path}")
    return a


def write_case(dirpath, p, x, v, extra_kv=None):
    os.makedirs(dirpath, exist_ok=True)
    write_params_kv(p, os.path.join(dirpath, "params.kv"), extra_kv)
    write_bin(os.path.join(dirpath, "in_x.bin"), x)
    write_bin(os.path.join(dirpath, "in_v.bin"), v)
    write_bin(os.path.join(dirpath, "in_type.bin"), np.zeros(p["n"], np.uint8), np.uint8)
    write_bin(os.path.join(dirpath, "in_r0.bin"), x)
