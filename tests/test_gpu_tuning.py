"""The collision's tile-shape autotuner: the shape it picks is one of the four, it waits for
cell-sorted slots (an uploaded state is in particle-id order until the first step re-sorts it),
and every shape gives the same state, bit for bit (a cell's collision does not depend on the
tiling)."""
import numpy as np
import pytest

from src_incompressible_openmp_b200.cases import poiseuille_params, uniform_state

pytestmark = pytest.mark.gpu


def _native():
    from src_incompressible_openmp_b200 import native
    if not native.device_available():
        pytest.fail("no CUDA device")
    return native


def test_every_collision_shape_gives_the_same_state():
    native = _native()
    p = poiseuille_params(96, 40, 14)
    x, v = uniform_state(p, 21)
    out = []
    with native.Context(p) as ctx:
        ctx.set_state(x, v)
        assert ctx.collide_shape() == -1
        ctx.step(0, 1)
        assert ctx.collide_shape() == -1  # the first step sorts the uploaded slots
        ctx.step(1, 2)
        assert 0 <= ctx.collide_shape() < native.COLLIDE_SHAPES  # picked by timing
        out.append(ctx.get_state())
    for shape in range(native.COLLIDE_SHAPES):
        with native.Context(p) as ctx:
            ctx.set_state(x, v)
            assert ctx.collide_shape(shape) == shape
            ctx.step(0, 3)
            assert ctx.collide_shape() == shape
            out.append(ctx.get_state())
    for xs, vs in out[1:]:
        assert np.array_equal(xs, out[0][0]) and np.array_equal(vs, out[0][1])


def test_shape_out_of_range_rejected():
    native = _native()
    p = poiseuille_params(16, 16, 5)
    with native.Context(p) as ctx:
        with pytest.raises(native.MpcdError):
            ctx.collide_shape(native.COLLIDE_SHAPES)


def test_contexts_of_different_density_keep_their_shared_memory():
    """A kernel's shared-memory limit is shared by all contexts of the process: a later context
    needing less must not lower it below an earlier one's need."""
    native = _native()
    dense = poiseuille_params(64, 32, 20)
    sparse = poiseuille_params(64, 32, 5)
    x, v = uniform_state(dense, 3)
    with native.Context(dense) as a:
        a.set_state(x, v)
        with native.Context(sparse) as b:
            xs, vs = uniform_state(sparse, 4)
            b.set_state(xs, vs)
            for shape in range(native.COLLIDE_SHAPES):
                a.collide_shape(shape)
                a.step(shape, 1)
                b.collide_shape(shape)
                b.step(shape, 1)
