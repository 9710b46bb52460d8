"""Parity of the CUDA path with the oracle at the benchmark workloads' own sizes.

The small cases of test_gpu_parity never reach the code paths that only large grids take.
These cases do:
  - the Poiseuille channel of 2048 x 512 cells at 10 particles per cell (10,485,760
    particles): the three-kernel count scan above 65,536 cells, which also packs the rank
    of every cell with N >= 2 (the index of its SRD sign draw), the rank-sort tiles of the
    cell index, zone launches over 10,660 + 10,712 zones ordered heaviest first in several
    waves, and the collision tile the autotuner picks at full size; checked phase by phase
    and as two whole teacher-forced steps;
  - the reference's own 50 x 50 case (25,000 particles): 20 teacher-forced steps, then a
    200-step free run whose metrics rows follow the oracle's;
  - a 512 x 256 channel with two dense blobs: the multi-block scan at 131,072 cells, cell
    segments above 2,048 particles (ranked from global memory), runs of cells split across
    rank tiles, and zones that overflow the shared-memory arena;
  - the 4096 x 1024 channel at 20 particles per cell (83,886,080 particles): one whole
    teacher-forced step.
The SRD sign ranks and the cell-index starts have no output of their own: they are checked
through the collision (each cell's sign comes from its rank) and the counts of the cell
fields, both bit-exact. Bars as in tests/parity_checks.py.
"""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state
from tests.parity_checks import (METRIC_KEYS, check_phases, check_teacher_forced_steps, native_or_fail,
                                 vclose)

pytestmark = pytest.mark.gpu


def test_channel_2048x512_phases(oracle):
    native = native_or_fail()
    p = poiseuille_params(2048, 512, 10)
    assert p["n"] == 10485760 and p["Nc"] == 1048576
    x, v = uniform_state(p, 1)
    check_phases(native, oracle, p, x, v, S=1)


def test_channel_2048x512_steps(oracle):
    native = native_or_fail()
    p = poiseuille_params(2048, 512, 10)
    x, v = uniform_state(p, 1)
    check_teacher_forced_steps(native, oracle, p, x, v, 2)


def test_poiseuille_50x50_teacher_forced_then_free_run(oracle):
    native = native_or_fail()
    p = poiseuille_params(50, 50, 10)
    assert p["n"] == 25000
    x, v = uniform_state(p, 1)
    check_teacher_forced_steps(native, oracle, p, x, v, 20)
    # free run: the device keeps its own state, the oracle its own, for 200 steps
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        xo, vo = x, v
        for s in range(1, 201):
            m = ctx.step(s - 1, 1, metrics=True)
            xo, vo, mo = oracle.step(p, xo, vo, s)
            for k in METRIC_KEYS:
                assert abs(m[k] - mo[k]) <= 1e-9 * max(1.0, abs(mo[k])), (s, k, m[k], mo[k])
            for ph in ("base", "shifted"):
                assert m[ph]["nParticlesMovedDense"] == mo[ph]["nParticlesMovedDense"], (s, ph)
        xg, vg = ctx.get_state()
    assert vclose(xg, xo) <= 1e-9 and vclose(vg, vo) <= 1e-9


def blob_state(p, seed):
    """Uniform state plus two blobs: 3 x 3 cells holding ~3,000 particles each, and 6 x 6 cells
    holding ~300 each."""
    x, v = uniform_state(p, seed)
    rng = np.random.default_rng(seed + 1)
    X = x.reshape(-1, 2)
    a = p["Lx"] / p["Nx"]
    k1, k2 = 27000, 10800
    X[:k1, 0] = 0.25 * p["Lx"] + 3 * a * (rng.random(k1) - 0.5)
    X[:k1, 1] = 0.5 * p["Ly"] + 3 * a * (rng.random(k1) - 0.5)
    X[k1:k1 + k2, 0] = 0.7 * p["Lx"] + 6 * a * (rng.random(k2) - 0.5)
    X[k1:k1 + k2, 1] = 0.3 * p["Ly"] + 6 * a * (rng.random(k2) - 0.5)
    return X.reshape(-1).copy(), v


def test_blob_512x256_multiblock_scan(oracle):
    native = native_or_fail()
    p = poiseuille_params(512, 256, 10)
    assert p["Nc"] > 65536
    x, v = blob_state(p, 71)
    X = x.reshape(-1, 2)
    cid = (np.floor(X[:, 0] / (p["Lx"] / p["Nx"])).astype(np.int64) * p["Ny"] +
           np.floor(X[:, 1] / (p["Ly"] / p["Ny"])).astype(np.int64))
    counts = np.bincount(cid, minlength=p["Nc"])
    assert counts.max() > 2048 and np.count_nonzero(counts > 200) >= 30  # the case reaches those paths
    check_phases(native, oracle, p, x, v, S=2)
    check_teacher_forced_steps(native, oracle, p, x, v, 2)


def test_channel_4096x1024_ppc20_step(oracle):
    native = native_or_fail()
    p = poiseuille_params(4096, 1024, 20)
    assert p["n"] == 83886080
    x, v = uniform_state(p, 1)
    check_teacher_forced_steps(native, oracle, p, x, v, 1)
