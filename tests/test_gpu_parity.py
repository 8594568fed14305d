"""GPU parity: libpfgpu (through its C ABI) against the reference's own
operands (golden fixtures) and against the oracle.

Tolerances (FP64 path):
* F(p) and J x: normwise relative error <= 1e-12, measured against the
  largest reference norm of the same timestep (near convergence F itself
  is tiny next to its flux terms, so a pointwise relative error is meaningless);
* M^-1 r: normwise relative error <= 1e-12;
* pressure after every timestep: max |p - p_ref| / max |p_ref| <= 1e-9, with
  identical Newton and GMRES iteration counts.
Mixed path (FP32 preconditioner and Jacobian storage): pressure within 1e-8
relative of the FP64 reference after every step.
"""

import numpy as np
import pytest

from parflow_b200 import cases

pytestmark = pytest.mark.gpu

CASES = cases.GOLDEN


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from parflow_b200 import solver

    return solver


def _npc(g):
    """Preconditioner dumps paired with a matvec dump (the preconditioner is
    set up at the matvec's pressure); a run on difference quotients has no
    matvec dumps."""
    return min(len(g["pc_in"]), len(g["mv_p"]))


def _pold(g, i):
    """Old pressure of matvec dump i (fixtures made after it was dumped)."""
    return g["mv_pold"][i] if "mv_pold" in g else None


def _skip_unavailable(name, precision):
    """PCMatrixType FullJacobian runs on the FP64 and FP32 multigrids only."""
    if precision == "mixed16" and cases.get(name).solver.pc_matrix_code():
        pytest.skip("FullJacobian is not available with the scaled FP16 multigrid")


def _scale_by_time(times, norms, floor):
    out = {}
    for t, n in zip(times, norms):
        out[t] = max(out.get(t, floor), n)
    return out


def _floor(prob):
    """Scale of the flux terms F sums (a unit-gradient vertical Darcy flux
    through every cell over one step): keeps the relative measure meaningful
    when F itself cancels to ~0 (equilibrium cases)."""
    kmax = float(np.max(prob.field3d(prob.perm)))
    return (prob.dt * prob.dx * prob.dy * kmax * prob.density * prob.gravity / prob.viscosity
            * np.sqrt(prob.ncells))


@pytest.mark.parametrize("name", CASES)
def test_residual_vs_reference(name, golden, gpu):
    g = golden(name)
    prob = cases.get(name)
    s = gpu.RichardsGPU(prob)
    norms = [np.linalg.norm(f) for f in g["fe_f"]]
    scale = _scale_by_time(g["fe_time"], norms, _floor(prob))
    for i in range(len(g["fe_p"])):
        s.set_time(g["fe_time"][i])
        f = s.nl_function_eval(g["fe_p"][i], g["fe_pold"][i], g["fe_sold"][i], g["fe_dt"][i])
        err = np.linalg.norm(f - g["fe_f"][i]) / scale[g["fe_time"][i]]
        assert err <= 1e-12, (name, i, err)


@pytest.mark.parametrize("name", CASES)
def test_jacobian_matvec_vs_reference(name, golden, gpu):
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name))
    for i in range(len(g["mv_x"])):
        s.set_time(g["mv_time"][i])
        y = s.jacobian_matvec(g["mv_p"][i], g["mv_dt"][i], g["mv_x"][i], _pold(g, i))
        err = np.linalg.norm(y - g["mv_y"][i]) / np.linalg.norm(g["mv_y"][i])
        assert err <= 1e-12, (name, i, err)


@pytest.mark.parametrize("name", CASES)
def test_preconditioner_vs_reference(name, golden, gpu):
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name))
    for i in range(_npc(g)):
        s.set_time(g["mv_time"][i])
        s.pc_setup(g["mv_p"][i], g["mv_dt"][i], _pold(g, i))
        z = s.pc_apply(g["pc_in"][i])
        err = np.linalg.norm(z - g["pc_out"][i]) / np.linalg.norm(g["pc_out"][i])
        assert err <= 1e-12, (name, i, err)


@pytest.mark.parametrize("name", CASES)
def test_first_preconditioner_vs_reference(name, golden, gpu):
    """The run's first preconditioner application, set up at the first
    function evaluation's pressure: also for difference-quotient runs (no
    matvec dumps), whose preconditioner matrix has no overland surface
    terms."""
    g = golden(name)
    if not len(g["pc_in"]):
        pytest.skip("no preconditioner dump")
    s = gpu.RichardsGPU(cases.get(name))
    s.set_time(g["fe_time"][0])
    s.pc_setup(g["fe_p"][0], g["fe_dt"][0], g["fe_pold"][0])
    z = s.pc_apply(g["pc_in"][0])
    err = np.linalg.norm(z - g["pc_out"][0]) / np.linalg.norm(g["pc_out"][0])
    assert err <= 1e-12, (name, err)


# normwise distance of the reduced-precision preconditioners from the
# reference's FP64 MGSemi output: FP32 storage and arithmetic, and the scaled
# FP16 operator (11-bit significands of A_ij / sqrt(A_ii A_jj))
PC_TOL = {"mixed": 1e-4, "mixed16": 5e-3}


@pytest.mark.parametrize("precision", ["mixed", "mixed16"])
@pytest.mark.parametrize("name", CASES)
def test_mixed_preconditioner_close(name, precision, golden, gpu):
    _skip_unavailable(name, precision)
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name), precision=precision)
    for i in range(_npc(g)):
        s.set_time(g["mv_time"][i])
        s.pc_setup(g["mv_p"][i], g["mv_dt"][i], _pold(g, i))
        z = s.pc_apply(g["pc_in"][i])
        err = np.linalg.norm(z - g["pc_out"][i]) / np.linalg.norm(g["pc_out"][i])
        assert err <= PC_TOL[precision], (name, i, err)


# the time-loop cases' steps come from pfgpu_run (tests/test_gpu_timeloop.py)
STEP_CASES = [c for c in CASES if c not in cases.TIME_LOOP]


@pytest.mark.parametrize("name", STEP_CASES)
def test_timesteps_vs_reference(name, golden, gpu):
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name))
    ps, sts = s.run()
    for t, (p, st) in enumerate(zip(ps, sts)):
        ref = g["press"][t + 1]
        err = np.abs(p - ref).max() / np.abs(ref).max()
        assert err <= 1e-9, (name, t, err)
        assert st.nonlin_iters == g["counts"][t, 0], (name, t)
        assert st.lin_iters == g["counts"][t, 1], (name, t)
        assert st.kinsol_status in (1, 2)


@pytest.mark.parametrize("precision", ["mixed", "mixed16"])
@pytest.mark.parametrize("name", STEP_CASES)
def test_mixed_timesteps_vs_reference(name, precision, golden, gpu):
    _skip_unavailable(name, precision)
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name), precision=precision)
    ps, sts = s.run()
    for t, p in enumerate(ps):
        ref = g["press"][t + 1]
        err = np.abs(p - ref).max() / np.abs(ref).max()
        assert err <= 1e-8, (name, t, err)


def test_mg_levels_match_oracle(gpu):
    from oracle.oracle import Oracle

    prob = cases.box_odd()
    assert gpu.RichardsGPU(prob).mg_levels() == Oracle(prob).mg().levels()


def test_config0_size_vs_oracle(gpu):
    """Config-0 size (64x64x32), two steps, against the oracle."""
    from oracle.oracle import Oracle
    from parflow_b200 import configs

    prob = configs.box(nsteps=2)
    ps_o, st_o = Oracle(prob).run()
    ps_g, st_g = gpu.RichardsGPU(prob).run()
    for t in range(2):
        err = np.abs(ps_g[t] - ps_o[t]).max() / np.abs(ps_o[t]).max()
        assert err <= 1e-9, (t, err)
        assert st_g[t].nonlin_iters == st_o[t].nni and st_g[t].lin_iters == st_o[t].nli


def test_deterministic(gpu):
    """Atomic-free kernels and fixed-order reductions: reruns are bitwise equal."""
    prob = cases.box_odd()
    a, _ = gpu.RichardsGPU(prob).run()
    b, _ = gpu.RichardsGPU(prob).run()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_device_pointers_match_host(gpu, golden):
    """torch CUDA tensors in ParFlow layout are used in place (no staging)."""
    import torch

    g = golden("box_small")
    s = gpu.RichardsGPU(cases.box_small())
    s.set_time(g["fe_time"][0])
    args = [gpu.pad(g[k][0]) for k in ("fe_p", "fe_pold", "fe_sold")]
    f_host = s.nl_function_eval(*[a[1:-1, 1:-1, 1:-1] for a in args], g["fe_dt"][0])
    dev = [torch.from_numpy(a).cuda() for a in args]
    out = torch.zeros_like(dev[0])
    import ctypes as C

    rc = s.lib.pfgpu_nl_function_eval(s.h, C.c_void_p(dev[0].data_ptr()),
                                      C.c_void_p(dev[1].data_ptr()), C.c_void_p(dev[2].data_ptr()),
                                      g["fe_dt"][0], C.c_void_p(out.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    f_dev = out.cpu().numpy()[1:-1, 1:-1, 1:-1]
    assert np.array_equal(f_dev, f_host)
    assert (out.cpu().numpy()[0] == 0).all()  # ghost frame written as zero


@pytest.mark.parametrize("name", ["overland_small", "overland_diff_small", "overland_flow_small"])
def test_preconditioner_grid_levels_vs_reference(name, golden, gpu, monkeypatch):
    """The grid-level setup and smoother kernels (the tail moved down to 16
    cells) against the reference's MGSemi output; with diffusive overland
    terms this includes the x_lower ghost column of the operator."""
    monkeypatch.setenv("PFGPU_TAIL_CELLS", "16")
    g = golden(name)
    s = gpu.RichardsGPU(cases.get(name))
    for i in range(_npc(g)):
        s.set_time(g["mv_time"][i])
        s.pc_setup(g["mv_p"][i], g["mv_dt"][i], _pold(g, i))
        z = s.pc_apply(g["pc_in"][i])
        err = np.linalg.norm(z - g["pc_out"][i]) / np.linalg.norm(g["pc_out"][i])
        assert err <= 1e-12, (name, i, err)


@pytest.mark.parametrize("precision", ["fp64", "mixed16"])
@pytest.mark.parametrize("kind", ["OverlandDiffusive", "OverlandFlow"])
def test_overland_types_vs_oracle(gpu, precision, kind):
    """Diffusive-wave and OverlandFlow overland flow on a 40 x 36 x 10
    hillslope (grid-level multigrid kernels), three steps against the oracle:
    FP64 within 1e-9 with identical Newton and GMRES counts, the mixed form
    within 1e-8."""
    from oracle.oracle import Oracle
    from parflow_b200 import configs
    from parflow_b200.problem import BC_OVERLAND, BC_OVERLAND_DIFF

    k = {"OverlandDiffusive": BC_OVERLAND_DIFF, "OverlandFlow": BC_OVERLAND}[kind]
    prob = configs.overland(nx=40, ny=36, nz=10, nsteps=3, seed=5, wt_depth=0.05,
                            mannings=3e-4, rain_steps=2, dry_steps=1, kind=k)
    ps_o, st_o = Oracle(prob).run()
    ps_g, st_g = gpu.RichardsGPU(prob, precision=precision).run()
    for t in range(3):
        err = np.abs(ps_g[t] - ps_o[t]).max() / np.abs(ps_o[t]).max()
        if precision == "fp64":
            assert err <= 1e-9, (t, err)
            assert st_g[t].nonlin_iters == st_o[t].nni and st_g[t].lin_iters == st_o[t].nli
        else:
            assert err <= 1e-8, (t, err)


def test_difference_quotient_counts_fevals(gpu, golden):
    """UseJacobian False: every GMRES product (and the line search's J p) is
    one more residual evaluation, as the reference counts them."""
    g = golden("dq_small")
    s = gpu.RichardsGPU(cases.get("dq_small"))
    _, sts = s.run()
    for t, st in enumerate(sts):
        assert st.fevals == g["counts"][t, 2], (t, st.fevals, g["counts"][t, 2])
        assert st.pc_solves == g["counts"][t, 4], (t, st.pc_solves)


@pytest.mark.parametrize("kind", ["OverlandKinematic", "OverlandDiffusive"])
def test_difference_quotient_overland_vs_oracle(gpu, kind):
    """KINSOL's difference-quotient J v with kinematic or diffusive overland
    flow (the preconditioner matrix without the surface terms, as the
    reference builds it under UseJacobian False; Krylov dimension 50 as the
    reference's tilted-V tests), 3 steps against the oracle: within 1e-9
    with identical Newton and GMRES counts."""
    from oracle.oracle import Oracle
    from parflow_b200 import configs
    from parflow_b200.problem import BC_OVERLAND_DIFF, BC_OVERLAND_KIN, SolverSettings

    k = {"OverlandKinematic": BC_OVERLAND_KIN, "OverlandDiffusive": BC_OVERLAND_DIFF}[kind]
    prob = configs.overland(nx=20, ny=18, nz=8, nsteps=3, dt=0.01, seed=11, wt_depth=0.05,
                            mannings=3e-4, rain_steps=2, dry_steps=1, kind=k,
                            solver=SolverSettings(use_jacobian=False, krylov_dim=50))
    ps_o, st_o = Oracle(prob).run()
    ps_g, st_g = gpu.RichardsGPU(prob).run()
    for t in range(3):
        err = np.abs(ps_g[t] - ps_o[t]).max() / np.abs(ps_o[t]).max()
        assert err <= 1e-9, (t, err)
        assert st_g[t].nonlin_iters == st_o[t].nni and st_g[t].lin_iters == st_o[t].nli


@pytest.mark.parametrize("precision", ["fp64", "mixed16"])
@pytest.mark.parametrize("max_iter", [0, 3])
def test_mg_max_iter_vs_oracle(gpu, max_iter, precision):
    """MGSemi.MaxIter 0 (the identity preconditioner; Krylov dimension 60)
    and 3 V-cycles per application, two steps against the oracle: FP64
    within 1e-9 with identical Newton and GMRES counts, mixed16 within
    1e-8.  MaxIter 2 is pinned to the reference by the golden
    mg_maxiter_small."""
    from oracle.oracle import Oracle
    from parflow_b200 import configs
    from parflow_b200.problem import SolverSettings

    prob = configs.hetero(nx=14, ny=12, nz=9, nsteps=2, dt=0.05, seed=31,
                          solver=SolverSettings(mg_max_iter=max_iter,
                                                krylov_dim=60 if max_iter == 0 else 25))
    ps_o, st_o = Oracle(prob).run()
    ps_g, st_g = gpu.RichardsGPU(prob, precision=precision).run()
    for t in range(2):
        err = np.abs(ps_g[t] - ps_o[t]).max() / np.abs(ps_o[t]).max()
        if precision == "fp64":
            assert err <= 1e-9, (t, err)
            assert st_g[t].nonlin_iters == st_o[t].nni and st_g[t].lin_iters == st_o[t].nli
        else:
            assert err <= 1e-8, (t, err)
