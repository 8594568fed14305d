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


def _advance_raw(members, nsteps):
    """pfgpu_ensemble_advance through the C ABI: (return code, per-member
    status, per-member per-step (Newton, GMRES) counts)."""
    import ctypes as C

    from parflow_b200 import lib as L

    n = len(members)
    lib = L.load()
    handles = (C.c_void_p * n)(*[g.h.value for g in members])
    dt = (C.c_double * n)(*[g.prob.dt for g in members])
    stats = (L.Stats * (n * nsteps))()
    status = (C.c_int * n)()
    rc = lib.pfgpu_ensemble_advance(handles, n, dt, nsteps, 0, stats, status)
    counts = [[(stats[m * nsteps + s].nonlin_iters, stats[m * nsteps + s].lin_iters)
               for s in range(nsteps)] for m in range(n)]
    return rc, list(status), counts


def test_ensemble_member_failure_as_alone(solver):
    """A member whose solves fail (Solver.Nonlinear.MaxIter 1) gets the
    retries with halved dt and the final failure pfgpu_advance gives it alone;
    the other members finish their steps as they would alone."""
    probs = _members()
    probs[1].solver.max_iter = 1
    alone = []
    for p in probs:
        g = _start(solver, p)
        rc = g.lib.pfgpu_advance(g.h, p.dt, NSTEPS, None)
        alone.append((rc, g.get_pressure()))
        g.close()
    assert alone[1][0] != 0 and all(a[0] == 0 for i, a in enumerate(alone) if i != 1)
    members = [_start(solver, p) for p in probs]
    rc, status, _ = _advance_raw(members, NSTEPS)
    assert rc == alone[1][0]
    for m, g in enumerate(members):
        assert status[m] == alone[m][0], m
        assert np.array_equal(g.get_pressure(), alone[m][1]), m
        g.close()


CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from parflow_b200 import configs
from parflow_b200.solver import RichardsGPU, ensemble_advance
probs = configs.ensemble(4, seed=5, nxy=(12, 16), nz=(8, 10), nsteps=3)
ms = []
for p in probs:
    g = RichardsGPU(p, precision=sys.argv[2])
    g.set_pressure(p.initial_pressure())
    g.set_time(p.start_time + p.dt)
    ms.append(g)
stats = ensemble_advance(ms, 3)
out = {"p": [g.get_pressure().tobytes().hex() for g in ms],
       "n": [[[s.nonlin_iters, s.lin_iters, s.fevals, s.backtracks] for s in m] for m in stats]}
json.dump(out, open(sys.argv[3], "w"))
"""


@pytest.mark.parametrize("precision", ["fp64", "mixed16"])
def test_ensemble_graph_equals_thread_pool(solver, tmp_path, precision):
    """One graph launch per ensemble timestep (the default) against the
    host-thread pool over the members (PFGPU_ENSEMBLE_GRAPH=0): bit for bit."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = []
    for flag in ("1", "0"):
        path = str(tmp_path / f"ens{flag}.json")
        env = dict(os.environ, PFGPU_ENSEMBLE_GRAPH=flag)
        subprocess.run([sys.executable, "-c", CHILD, root, precision, path], env=env, check=True,
                       timeout=600)
        res.append(json.load(open(path)))
    assert res[0]["n"] == res[1]["n"]
    assert res[0]["p"] == res[1]["p"]
