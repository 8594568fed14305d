"""The GPU nonlinear-solver module inside ParFlow itself.

oracle/_ref/bin/parflow_gpu is the unmodified reference build with the module
of parflow_b200/pfmodule/kinsol_gpu_nonlin_solver.c linked in (ld --wrap on
the KINSol module's functions).  ParFlow's own driver runs the whole problem:
input database, BCPressure, the time loop of AdvanceRichards, saturation and
PFB output; only the nonlinear solve of each step moves to the GPU when the
run sets Solver.Nonlinear.GPU True.

* CPU (no marker): without the key the binary is the reference: its
  pressures equal the golden fixtures bit for bit, with the same counts.
* GPU: with the key, the pressure after every step matches the reference's
  golden pressures within 1e-9 (FP64; 1e-8 for the mixed forms) with the
  same Newton and GMRES counts (FP64), and the face velocities ParFlow writes
  (velx / vely / velz) match the reference's within 1e-9 of their scale.
"""

import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.refrun import BIN, kinsol_counts
from parflow_b200 import cases
from parflow_b200.pfb import read_pfb

EXE = os.path.join(BIN, "parflow_gpu")


def _need_exe():
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/bin/parflow_gpu missing (oracle/ref.mk target gpu, built "
                    "where the ParFlow sources are)")


def _run(name, gpu=None):
    prob = cases.get(name)
    wd = tempfile.mkdtemp(prefix="pfgpu_mod_")
    run = prob.to_reference(wd, "m", dump_interval=cases.DUMP.get(name, 1), gpu=gpu)
    r = subprocess.run([EXE, run], cwd=wd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    nfiles = 1
    while os.path.exists(os.path.join(wd, f"{run}.out.press.{nfiles:05d}.pfb")):
        nfiles += 1
    press = [read_pfb(os.path.join(wd, f"{run}.out.press.{t:05d}.pfb")) for t in range(1, nfiles)]
    vel = {}
    for key in ("velx", "vely", "velz"):
        f = [os.path.join(wd, f"{run}.out.{key}.{t:05d}.pfb") for t in range(1, nfiles)]
        if all(os.path.exists(x) for x in f):
            vel[key] = [read_pfb(x) for x in f]
    counts = kinsol_counts(open(os.path.join(wd, f"{run}.out.kinsol.log")).read())
    return prob, press, vel, counts


@pytest.mark.parametrize("name", ["box_small", "vel_small", "halving_small"])
def test_wrapped_build_without_gpu_is_the_reference(name, golden):
    _need_exe()
    g = golden(name)
    prob, press, _, counts = _run(name)
    assert len(press) == len(g["press"]) - 1
    for t, p in enumerate(press, start=1):
        assert np.array_equal(p, g["press"][t]), (name, t)
    assert np.array_equal(counts[:, :2], g["counts"][:, :2])


GPU_CASES = ["box_small", "box_odd", "hetero_small", "walker2_small", "seepage_small",
             "overland_small", "tfg_small", "vel_small", "vel_overland_small", "wjacobi_small",
             "krtable_spline_small", "growth_small", "halving_small", "restart_small",
             "inexact_small", "rbgs_nonsym_small", "flow_barrier_small", "fulljac_small",
             "fulljac_overland_small", "dq_overland_flow_small", "dirichlet_top_small",
             "mg_maxiter_small", "mg_minn_small", "spinup_small", "spinup_damp_small"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", GPU_CASES)
def test_parflow_with_gpu_module_fp64(name, golden):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    _need_exe()
    g = golden(name)
    prob, press, vel, counts = _run(name, gpu="FP64")
    # ParFlow's own time loop: growth, transition cuts, dt halving after a
    # failed GPU solve (its kinsol.log rows include the failed attempts)
    assert len(press) == len(g["press"]) - 1
    for t, p in enumerate(press, start=1):
        ref = g["press"][t]
        err = float(np.abs(p - ref).max() / np.abs(ref).max())
        assert err <= 1e-9, (name, t, err)
    assert np.array_equal(counts[:, :2], g["counts"][:, :2]), (counts[:, :2], g["counts"][:, :2])
    for key, vs in vel.items():
        if key not in g:
            continue
        for t, v in enumerate(vs):
            ref = g[key][t]
            scale = float(np.abs(ref).max())
            if key == "velz" and "qx_overland" in g:
                # the overland top face carries the near-cancelling surface
                # fluxes (ke - kw) / dx + (kn - ks) / dy: their size is the scale
                scale = max(scale, float(np.abs(g["qx_overland"][t]).max()) / prob.dx,
                            float(np.abs(g["qy_overland"][t]).max()) / prob.dy)
            err = float(np.abs(v - ref).max() / max(scale, 1e-300))
            assert err <= 1e-9, (name, key, t + 1, err)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["Mixed", "Mixed16"])
def test_parflow_with_gpu_module_mixed(precision, golden):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    _need_exe()
    g = golden("hetero_small")
    _, press, _, _ = _run("hetero_small", gpu=precision)
    for t, p in enumerate(press, start=1):
        ref = g["press"][t]
        err = float(np.abs(p - ref).max() / np.abs(ref).max())
        assert err <= 1e-8, (precision, t, err)
