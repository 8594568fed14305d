"""The block-shape autotuner (pfgpu_autotune) through the C ABI: the shapes it
picks are valid launch shapes, a second handle of the same size takes them
from the cache, and a solve with tuned shapes is bitwise equal to one with the
built-in heuristic (every cell's arithmetic is independent of the block)."""

import numpy as np
import pytest

from parflow_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _valid(shape, threads):
    bx, by = shape
    if (bx, by) == (0, 0):
        return True
    return bx % 32 == 0 and by >= 1 and bx * by <= threads


@pytest.mark.parametrize("precision", ["fp64", "mixed16"])
def test_autotuned_solve_bitwise_equals_heuristic(solver, precision):
    prob = configs.ensemble_member(5, nsteps=2, nxy=(96,), nz=(16,))
    a = solver.RichardsGPU(prob, precision=precision)
    a.set_pressure(prob.initial_pressure())
    shapes = a.autotune(reps=3)
    assert _valid(shapes["residual"], 256) and _valid(shapes["matvec"], 256)
    assert _valid(shapes["jacobian"], 128)
    ps_a, st_a = a.run(2)
    b = solver.RichardsGPU(prob, precision=precision)
    ps_b, st_b = b.run(2)
    for x, y in zip(ps_a, ps_b):
        assert np.array_equal(x, y)
    assert [s.lin_iters for s in st_a] == [s.lin_iters for s in st_b]
    # a second handle of the same size takes the cached choice
    c = solver.RichardsGPU(prob, precision=precision)
    assert c.autotune(reps=3) == shapes
    for g in (a, b, c):
        g.close()


def test_forced_shapes_bitwise_equal(solver):
    """Tuned shapes give the same residual and matvec as the heuristic, bit
    for bit."""
    prob = configs.box(nx=40, ny=12, nz=6, nsteps=1, seed=4)
    g = solver.RichardsGPU(prob)
    p = prob.initial_pressure()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(prob.shape)
    f0 = g.nl_function_eval(p, p, g.saturation(p), prob.dt)
    y0 = g.jacobian_matvec(p, prob.dt, x)
    g.autotune(reps=2)
    f1 = g.nl_function_eval(p, p, g.saturation(p), prob.dt)
    y1 = g.jacobian_matvec(p, prob.dt, x)
    assert np.array_equal(f0, f1) and np.array_equal(y0, y1)
    g.close()
