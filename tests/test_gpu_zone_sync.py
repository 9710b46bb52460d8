"""The phase-synchronous zone kernels (several zones per block, a barrier between phases) against
the one-zone-per-block kernels: the same state after several steps, for each block width of the
FP64 kernel and for the fast form's decision kernel."""
import os

import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    return native


def _run(native, p, x, v, form, steps, env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        with native.Context(p, form=form) as ctx:
            ctx.set_state(x, v)
            ctx.step(0, steps)
            return ctx.get_state()
    finally:
        for k, val in old.items():
            if val is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = val


def test_fp64_zone_pass_block_widths_agree():
    native = _native()
    p = poiseuille_params(210, 130, 10)
    x, v = uniform_state(p, 21)
    ref = _run(native, p, x, v, "f64", 4, {"MPCD_ZONE_SYNC_WARPS": "0"})
    for w in ("4", "8", "16"):
        got = _run(native, p, x, v, "f64", 4, {"MPCD_ZONE_SYNC_WARPS": w})
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), w


def test_fast_zone_decisions_block_widths_agree():
    native = _native()
    p = poiseuille_params(210, 130, 16)
    x, v = uniform_state(p, 22)
    a = _run(native, p, x, v, "fast", 8, {"MPCD_FAST_ZONE_WARPS": "4"})
    b = _run(native, p, x, v, "fast", 8, {})
    assert not np.isnan(a[1]).any()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
