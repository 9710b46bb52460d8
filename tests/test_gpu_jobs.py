"""mpcd_run_jobs: independent jobs with host buffers, their copies overlapped with the steps of
the neighbouring jobs, give exactly the states of mpcd_set_state + mpcd_step + mpcd_get_state
per job (consecutive step numbers), in both state forms, from pageable or page-locked host
memory, with a job's output written over its own input or not."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no CUDA device")
    return native


def _serial(native, p, form, xs, vs, step0, nsteps):
    out = []
    with native.Context(p, form=form) as ctx:
        for j, (x, v) in enumerate(zip(xs, vs)):
            ctx.set_state(x, v)
            ctx.step(step0 + j * nsteps, nsteps)
            out.append(ctx.get_state())
    return out


@pytest.mark.parametrize("form", ["f64", "f32"])
def test_jobs_match_serial_calls(form):
    native = _native()
    p = poiseuille_params(96, 40, 10)
    states = [uniform_state(p, 30 + j) for j in range(5)]
    xs = [s[0] for s in states]
    vs = [s[1] for s in states]
    want = _serial(native, p, form, xs, vs, 4, 3)
    with native.Context(p, form=form) as ctx:
        xo, vo = ctx.run_jobs(xs, vs, 4, 3)
    for j in range(5):
        assert np.array_equal(xo[j], want[j][0]) and np.array_equal(vo[j], want[j][1]), j


def test_jobs_in_place_from_page_locked_memory():
    native = _native()
    p = poiseuille_params(64, 32, 12)
    states = [uniform_state(p, 50 + j) for j in range(4)]
    want = _serial(native, p, "f64", [s[0] for s in states], [s[1] for s in states], 0, 2)
    bufs = [(native.PinnedArray(2 * p["n"]), native.PinnedArray(2 * p["n"])) for _ in states]
    try:
        for (hx, hv), (x, v) in zip(bufs, states):
            hx.array[:] = x
            hv.array[:] = v
        xs = [b[0].array for b in bufs]
        vs = [b[1].array for b in bufs]
        with native.Context(p) as ctx:
            ctx.run_jobs(xs, vs, 0, 2, xs, vs)  # each job's result over its own input
        for j in range(4):
            assert np.array_equal(xs[j], want[j][0]) and np.array_equal(vs[j], want[j][1]), j
    finally:
        for hx, hv in bufs:
            hx.close()
            hv.close()


def test_jobs_then_ordinary_steps():
    """After run_jobs the context holds the last job's state and keeps stepping from it."""
    native = _native()
    p = poiseuille_params(48, 32, 8)
    states = [uniform_state(p, 70 + j) for j in range(2)]
    with native.Context(p) as ctx:
        ctx.run_jobs([s[0] for s in states], [s[1] for s in states], 0, 2)
        ctx.step(4, 3)
        got = ctx.get_state()
    with native.Context(p) as ctx:
        ctx.set_state(*states[1])
        ctx.step(2, 2)
        ctx.step(4, 3)
        want = ctx.get_state()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_jobs_argument_errors():
    native = _native()
    p = poiseuille_params(16, 16, 5)
    x, v = uniform_state(p, 1)
    with native.Context(p) as ctx:
        assert ctx.run_jobs([], [], 0, 1) == ([], [])
        with pytest.raises(ValueError):
            ctx.run_jobs([x[:-2]], [v], 0, 1)
        assert native.lib().mpcd_run_jobs(ctx.h, 1, None, None, 0, 1, None, None) == 1  # MPCD_ERR_INVALID_ARG
        assert b"null" in native.lib().mpcd_last_error()
