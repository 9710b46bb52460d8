"""The ensemble leg's flux (bench._ensemble_flux): Qx = meanUx * Ly with meanUx the mean over cells
of the cell mean vx (src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:124-126),
averaged over the states it samples; checked on CPU with a stand-in batch whose states are known."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from src_incompressible_openmp_b200.cases import poiseuille_params  # noqa: E402


class _Member:
    def __init__(self, x, vs):
        self.x, self.vs, self.k = x, vs, 0

    def get_state(self):
        v = self.vs[min(self.k, len(self.vs) - 1)]
        return self.x, v


class _Batch:
    """Each step call moves every member to its next velocity field."""

    def __init__(self, members):
        self.members = members
        self.calls = []

    def step(self, s0, k):
        self.calls.append((s0, k))
        for m in self.members:
            m.k += 1

    def member(self, i):
        return self.members[i]


def _state(p, extra, ux_of_row):
    """One particle at the centre of every cell, vx by row, plus one more in each cell of extra."""
    ax, ay = p["Lx"] / p["Nx"], p["Ly"] / p["Ny"]
    ix, iy = np.meshgrid(np.arange(p["Nx"]), np.arange(p["Ny"]), indexing="ij")
    ix, iy = ix.ravel(), iy.ravel()
    ix = np.concatenate([ix, ix[extra]])
    iy = np.concatenate([iy, iy[extra]])
    x = np.empty(2 * ix.size)
    x[0::2] = (ix + 0.5) * ax
    x[1::2] = (iy + 0.5) * ay
    v = np.zeros_like(x)
    v[0::2] = ux_of_row(iy)
    return x, v


def test_flux_is_mean_cell_velocity_times_height():
    rng = np.random.default_rng(3)
    reps = [(poiseuille_params(12, 8, 1), 0), (poiseuille_params(9, 5, 1), 1)]
    members = []
    want = []
    for p, _ in reps:
        # the state before the first step, then the three sampled after each step call
        fields = [lambda iy, a=a: a * (iy + 1.0) for a in (0.5, 1.0, 2.0, 4.0)]
        extra = rng.integers(0, p["Nc"], 7)
        x, _ = _state(p, extra, fields[0])
        vs = [_state(p, extra, f)[1] for f in fields]
        # every cell holds particles of one row only, so each cell mean is its row's vx
        mean_ux = [np.mean(f(np.arange(p["Ny"]).repeat(p["Nx"]))) for f in fields[1:]]
        members.append(_Member(x, vs))
        want.append(np.mean(mean_ux) * p["Ly"])
    B = _Batch(members)
    q = bench._ensemble_flux(B, reps, 100, 3, 10)
    assert B.calls == [(100, 10), (110, 10), (120, 10)]
    assert np.allclose(q, want, rtol=1e-12)
