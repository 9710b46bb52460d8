"""mpcd_cell_fields_static (the entry point that allocates no device memory) against
mpcd_cell_fields on the same state.

The caller here owns every device buffer (torch tensors stand in for the caller's pool); the
entry point itself only uses its static scratch array. Counts must match exactly; the other
fields within the 1e-12 relative bar of the velocity checks (its sums are accumulated with
atomics, in a different order).

The cases: two calls in a row on a changing state; a grid of exactly the static maximum
(every entry of the array in use); a smaller grid after a larger one (sums left beyond the
new grid must not leak in); only N, Ux and Uy requested (the path that skips the peculiar
speeds); no particles at all; and a call in a fresh process, where the first call does the
per-device set-up, run as a child process so it does not depend on what ran before.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from src_incompressible_openmp_b200 import _abi
from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

REL = 1e-12
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def vclose(a, b):
    d = np.abs(a - b) / np.maximum(1.0, np.abs(b))
    return float(d.max()) if d.size else 0.0


def test_rejects_grids_beyond_the_static_maximum():
    """Rejected before any device work, so this runs without a GPU."""
    from src_incompressible_openmp_b200 import native

    p = poiseuille_params(2048, 513, 1)  # 1,050,624 cells > 1,048,576
    with pytest.raises(native.MpcdError) as e:
        native.cell_fields_static(p, 0, 0, 0, 1.0, {})
    assert e.value.code == 6 and "static scratch maximum" in str(e.value)


def _native():
    from src_incompressible_openmp_b200 import native

    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def _rho_target(p):
    return p["gamma"] / ((p["Lx"] / p["Nx"]) * (p["Ly"] / p["Ny"]))


def static_fields(native, p, xs, vs, names=None):
    """Runs the static entry point on device copies of (xs, vs); returns the requested fields."""
    import torch

    dev = torch.device("cuda:0")
    Nc = p["Nc"]
    names = list(names or (["N"] + list(_abi.FIELD_NAMES)))
    dx = torch.from_numpy(xs).to(dev)
    dv = torch.from_numpy(vs).to(dev)
    out = {}
    for k in names:
        if k == "N":
            out[k] = torch.full((Nc,), -1, dtype=torch.int32, device=dev)
        else:
            out[k] = torch.full((Nc,), np.nan, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    n = xs.size // 2
    native.cell_fields_static(p, dx.data_ptr() if n else 0, dv.data_ptr() if n else 0, n, _rho_target(p),
                              {k: t.data_ptr() for k, t in out.items()}, stream.cuda_stream)
    stream.synchronize()
    return {k: t.cpu().numpy() for k, t in out.items()}


def check_against_context(native, p, xs, vs, got, label):
    with native.Context(p) as ctx:
        ctx.set_state(xs, vs)
        want = ctx.cell_fields(_rho_target(p))
    assert np.array_equal(got["N"], want["N"]), f"{label}: counts"
    for k in got:
        if k != "N":
            assert vclose(got[k], want[k]) <= REL, f"{label}: {k}"


@pytest.mark.gpu
def test_static_fields_match_context_fields_twice():
    native = _native()
    p = poiseuille_params(64, 48, 10)
    x, v = uniform_state(p, 41)
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        for call in range(2):
            ctx.step(call, 1)  # a different state for each of the two calls
            xs, vs = ctx.get_state()
            want = ctx.cell_fields(_rho_target(p))
            got = static_fields(native, p, xs, vs)
            assert np.array_equal(got["N"], want["N"]), f"call {call}: counts"
            for k in _abi.FIELD_NAMES:
                assert vclose(got[k], want[k]) <= REL, f"call {call}: {k}"


@pytest.mark.gpu
def test_static_maximum_then_smaller_grid():
    """2048 x 512 = 1,048,576 cells fills the whole array; the 96 x 40 grid after it must not
    see the larger grid's sums."""
    native = _native()
    big = poiseuille_params(2048, 512, 2)
    assert big["Nc"] == 1048576
    xb, vb = uniform_state(big, 42)
    check_against_context(native, big, xb, vb, static_fields(native, big, xb, vb), "2048x512")
    small = poiseuille_params(96, 40, 10)
    xs, vs = uniform_state(small, 43)
    check_against_context(native, small, xs, vs, static_fields(native, small, xs, vs), "96x40 after 2048x512")


@pytest.mark.gpu
def test_static_fields_subset_and_empty():
    native = _native()
    p = poiseuille_params(50, 30, 8)
    x, v = uniform_state(p, 44)
    got = static_fields(native, p, x, v, names=("N", "Ux", "Uy"))
    check_against_context(native, p, x, v, got, "N, Ux, Uy only")
    got = static_fields(native, p, np.zeros(0), np.zeros(0))  # n = 0: no particles
    assert np.array_equal(got["N"], np.zeros(p["Nc"], np.int32))
    for k in _abi.FIELD_NAMES:
        if k not in ("rho", "Pvir", "P", "rhoTarget"):
            assert np.array_equal(got[k], np.zeros(p["Nc"])), k


_FRESH = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from src_incompressible_openmp_b200 import native
from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state
from tests.test_zz_no_alloc import static_fields, check_against_context
p = poiseuille_params(40, 30, 10)
x, v = uniform_state(p, 45)
got = static_fields(native, p, x, v)  # the first call of this process: it does the set-up
check_against_context(native, p, x, v, got, "fresh process")
got = static_fields(native, p, x, v)
check_against_context(native, p, x, v, got, "fresh process, second call")
print("fresh ok")
"""


@pytest.mark.gpu
def test_static_fields_in_a_fresh_process():
    _native()
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout + r.stderr
