"""Colour-split storage of x and b on the multigrid grid levels.

By default every grid level keeps x and b as two colour blocks (cells of
parity (i+j+k) & 1 at (i >> 1) + hx (j + ny k) of their block), so that a
red/black sweep touches one colour's lines only; PFGPU_SPLIT=0 keeps the
natural interleaved layout.  The arithmetic is the same, so preconditioner
outputs and whole Newton solves must be bitwise identical in every precision,
for even and odd extents and with the tail boundary moved.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _problems():
    return {
        "box_small": cases.box_small(),
        "box_odd": configs.box(nx=33, ny=17, nz=9, nsteps=2),
        "box_flat": configs.box(nx=21, ny=19, nz=1, nsteps=2),
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=2),
    }


def _pc(solver, prob, precision, monkeypatch, split, tail="16"):
    monkeypatch.setenv("PFGPU_SPLIT", split)
    monkeypatch.setenv("PFGPU_TAIL_CELLS", tail)
    s = solver.RichardsGPU(prob, precision=precision)
    rng = np.random.default_rng(13)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    s.pc_setup(p, prob.dt)
    z = s.pc_apply(r)
    s.close()
    return z


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed16"])
@pytest.mark.parametrize("name", ["box_small", "box_odd", "box_flat", "hetero_96"])
def test_split_pc_bitwise_equal(solver, monkeypatch, name, precision):
    prob = _problems()[name]
    z_split = _pc(solver, prob, precision, monkeypatch, "1")
    z_nat = _pc(solver, prob, precision, monkeypatch, "0")
    assert np.isfinite(z_split).all() and np.abs(z_split).max() > 0
    assert np.array_equal(z_split, z_nat)
    # default tail boundary (the last split level restricts into the tail)
    assert np.array_equal(_pc(solver, prob, precision, monkeypatch, "1", "1024"),
                          _pc(solver, prob, precision, monkeypatch, "0", "1024"))


@pytest.mark.parametrize("precision", ["fp64", "mixed16"])
def test_split_newton_bitwise_equal(solver, monkeypatch, precision):
    prob = _problems()["hetero_96"]
    out = {}
    for split in ("1", "0"):
        monkeypatch.setenv("PFGPU_SPLIT", split)
        s = solver.RichardsGPU(prob, precision=precision)
        s.set_pressure(prob.initial_pressure())
        s.advance(prob.nsteps, prob.dt)
        out[split] = s.get_pressure()
        s.close()
    assert np.array_equal(out["1"], out["0"])
