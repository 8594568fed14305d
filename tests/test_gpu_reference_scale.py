"""GPU parity at scale against the unmodified reference build.

The heterogeneous box of the bench workload (sigma lnK 1.5, correlation
32x32x4 cells, per-cell alpha +-20 %, dt 0.05 h) on a 256x256x50 grid
(3.3M cells, the same physics as the 512x512x50 bench grid): the reference's
OpenMP build (oracle/_ref/bin/parflow_omp, every host thread) runs three
timesteps from the initial condition and writes its pressure after each;
every GPU form runs the same three steps through the C ABI.

Tolerances, per step:
* FP64: max |p - p_ref| / max |p_ref| <= 1e-9, Newton and GMRES counts equal
  to the reference's;
* mixed (FP32 multigrid and Jacobian storage) and mixed16 (scaled FP16
  multigrid operator): max relative difference <= 1e-8.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ, STEPS = 256, 256, 50, 3


@pytest.fixture(scope="module")
def reference_run():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from oracle import refrun
    from parflow_b200 import configs

    if refrun.binary("parflow_omp") is None:
        pytest.skip("reference build oracle/_ref/bin/parflow_omp missing "
                    "(made by oracle/ref.mk where the ParFlow sources are)")
    prob = configs.hetero(nx=NX, ny=NY, nz=NZ, nsteps=STEPS)
    res = refrun.run(prob, STEPS, dump=True)
    assert res["counts"].shape[0] == STEPS
    return prob, res


@pytest.mark.parametrize("precision,tol,counts", [("fp64", 1e-9, True),
                                                 ("mixed", 1e-8, False),
                                                 ("mixed16", 1e-8, False)])
def test_hetero_256x256x50_vs_reference(reference_run, precision, tol, counts):
    from parflow_b200.solver import RichardsGPU

    prob, res = reference_run
    g = RichardsGPU(prob, precision=precision)
    g.set_pressure(prob.initial_pressure())
    plan = prob.time_plan()
    for n in range(STEPS):
        t, dt = plan[n]
        g.set_time(t)
        st = g.advance(1, dt)[0]
        p = g.get_pressure()
        ref = res["press"][n]
        err = float(np.abs(p - ref).max() / np.abs(ref).max())
        assert err <= tol, (precision, n + 1, err)
        if counts:
            assert (st.nonlin_iters, st.lin_iters) == tuple(int(v) for v in res["counts"][n, :2]), \
                (n + 1, st.nonlin_iters, st.lin_iters, res["counts"][n, :2])
    g.close()
