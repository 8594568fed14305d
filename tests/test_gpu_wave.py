"""The wavefront red/black/red smoother (k_rbr_wave) against the per-colour
sweep kernels.

PFGPU_WAVE_CELLS selects, at handle creation, the grid levels the wavefront
kernel smooths: 0 = every grid level, a huge value = none.  PFGPU_TAIL_CELLS
= 16 keeps all but the last few levels on grid kernels, so that the small
fixtures have many wavefront levels, including ones with a single plane and
odd extents.  Both smoothers perform the same per-cell arithmetic in the same
sequential order, so the preconditioner output and whole Newton solves must
be bitwise identical.
"""

import numpy as np
import pytest

from parflow_b200 import cases, configs

pytestmark = pytest.mark.gpu

ALL, NONE = "0", str(1 << 62)


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
        "box_64": configs.box(nsteps=2),
        "hetero_96": configs.hetero(nx=96, ny=80, nz=20, nsteps=2),
    }


def _env(monkeypatch, cells):
    monkeypatch.setenv("PFGPU_WAVE_CELLS", cells)
    monkeypatch.setenv("PFGPU_TAIL_CELLS", "16")
    monkeypatch.setenv("PFGPU_SPLIT", "0")  # the wavefront kernel reads the natural layout


def _pc(solver, prob, precision, monkeypatch, cells):
    _env(monkeypatch, cells)
    s = solver.RichardsGPU(prob, precision=precision)
    rng = np.random.default_rng(7)
    p = prob.initial_pressure() + 0.1 * rng.standard_normal(prob.shape)
    r = rng.standard_normal(prob.shape)
    s.pc_setup(p, prob.dt)
    z = s.pc_apply(r)
    z2 = s.pc_apply(r)  # control words reset by the kernel itself
    s.close()
    assert np.array_equal(z, z2)
    return z


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["box_small", "box_odd", "box_64", "hetero_96"])
def test_wave_pc_bitwise_equal(solver, monkeypatch, name, precision):
    prob = _problems()[name]
    z_wave = _pc(solver, prob, precision, monkeypatch, ALL)
    z_ref = _pc(solver, prob, precision, monkeypatch, NONE)
    assert np.isfinite(z_wave).all() and np.abs(z_wave).max() > 0
    assert np.array_equal(z_wave, z_ref)


def _advance(solver, prob, precision, monkeypatch, cells):
    _env(monkeypatch, cells)
    s = solver.RichardsGPU(prob, precision=precision)
    s.set_pressure(prob.initial_pressure())
    stats = s.advance(prob.nsteps, prob.dt)
    p = s.get_pressure()
    s.close()
    return p, stats


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wave_newton_bitwise_equal(solver, monkeypatch, precision):
    prob = _problems()["hetero_96"]
    p_wave, _ = _advance(solver, prob, precision, monkeypatch, ALL)
    p_ref, _ = _advance(solver, prob, precision, monkeypatch, NONE)
    assert np.array_equal(p_wave, p_ref)
