"""mpcd_cell_fields_static (the entry point that allocates no device memory) against
mpcd_cell_fields on the same state.

The caller here owns every device buffer (torch tensors stand in for the caller's pool); the
entry point itself only uses its static scratch array. Counts must match exactly; the other
fields within the 1e-12 relative bar of the velocity checks (its sums are accumulated with
atomics, in a different order). This file is collected last on purpose: it must pass both in
a fresh process, where its first call performs the per-device set-up, and after the other tests.
"""
import numpy as np
import pytest

from src_incompressible_openmp_b200 import _abi
from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

REL = 1e-12


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


@pytest.mark.gpu
def test_static_fields_match_context_fields_twice():
    import torch

    from src_incompressible_openmp_b200 import native

    if not native.device_available():
        pytest.fail("no sm_100 device: the CUDA path has no CPU fallback")
    p = poiseuille_params(64, 48, 10)
    rho_t = p["gamma"] / ((p["Lx"] / p["Nx"]) * (p["Ly"] / p["Ny"]))
    x, v = uniform_state(p, 41)
    Nc = p["Nc"]
    dev = torch.device("cuda:0")
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        for call in range(2):
            ctx.step(call, 1)  # a different state for each of the two calls
            xs, vs = ctx.get_state()
            want = ctx.cell_fields(rho_t)
            dx = torch.from_numpy(xs).to(dev)
            dv = torch.from_numpy(vs).to(dev)
            out = {k: torch.full((Nc,), np.nan, dtype=torch.float64, device=dev) for k in _abi.FIELD_NAMES}
            out["N"] = torch.full((Nc,), -1, dtype=torch.int32, device=dev)
            stream = torch.cuda.current_stream(dev)
            native.cell_fields_static(p, dx.data_ptr(), dv.data_ptr(), p["n"], rho_t,
                                      {k: t.data_ptr() for k, t in out.items()}, stream.cuda_stream)
            stream.synchronize()
            got = {k: t.cpu().numpy() for k, t in out.items()}
            assert np.array_equal(got["N"], want["N"]), f"call {call}: counts"
            for k in _abi.FIELD_NAMES:
                assert vclose(got[k], want[k]) <= REL, f"call {call}: {k}"
