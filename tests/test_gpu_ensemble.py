"""Ensemble stepping (pfgpu_ensemble_advance): members advanced concurrently,
each on its own stream, must give exactly what each member gives when run
alone, and match the oracle within the FP64 timestep bound (1e-9 max-relative
pressure, identical Newton and GMRES counts)."""

import numpy as np
import pytest

from parflow_b200 import configs

pytestmark = pytest.mark.gpu

NSTEPS = 3


def _members():
    return configs.ensemble(4, seed=5, nxy=(12, 16), nz=(8, 10), nsteps=NSTEPS)


@pytest.fixture(scope="module")
def solver():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver as s

    return s


def _start(solver, prob, precision="fp64"):
    g = solver.RichardsGPU(prob, precision=precision)
    g.set_pressure(prob.initial_pressure())
    g.set_time(prob.start_time + prob.dt)
    return g


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_equals_members_alone(solver, precision):
    probs = _members()
    alone = []
    for p in probs:
        g = _start(solver, p, precision)
        st = g.advance(NSTEPS)
        alone.append((g.get_pressure(), [(s.nonlin_iters, s.lin_iters) for s in st]))
        g.close()
    members = [_start(solver, p, precision) for p in probs]
    stats = solver.ensemble_advance(members, NSTEPS, threads=0)
    for m, g in enumerate(members):
        assert np.array_equal(g.get_pressure(), alone[m][0]), m
        assert [(s.nonlin_iters, s.lin_iters) for s in stats[m]] == alone[m][1]
        g.close()


def test_ensemble_vs_oracle(solver):
    from oracle.oracle import Oracle

    probs = _members()
    members = [_start(solver, p) for p in probs]
    stats = solver.ensemble_advance(members, NSTEPS, threads=2)
    for m, (p, g) in enumerate(zip(probs, members)):
        orc = Oracle(p)
        ps_o, st_o = orc.run(NSTEPS)
        p_g = g.get_pressure()
        err = np.abs(p_g - ps_o[-1]).max() / np.abs(ps_o[-1]).max()
        assert err <= 1e-9, (m, err)
        assert [s.nonlin_iters for s in stats[m]] == [s.nni for s in st_o]
        assert [s.lin_iters for s in stats[m]] == [s.nli for s in st_o]
        g.close()


def test_ensemble_rejects_bad_arguments(solver):
    import ctypes as C

    from parflow_b200 import lib as L

    g = _start(solver, _members()[0])
    lib = L.load()
    handles = (C.c_void_p * 1)(g.h.value)
    dt = (C.c_double * 1)(-1.0)
    status = (C.c_int * 1)()
    assert lib.pfgpu_ensemble_advance(handles, 1, dt, 1, 0, None, status) == -1
    assert "dt" in L.last_error()
    g.close()
