"""The benchmark workloads as :class:`RichardsProblem` instances.

* ``box``  (config 0): plain FP64 Richards box, 64x64x32, lognormal K
  (geometric mean 0.01 m/h, sigma_lnK 1, correlation 8 cells), VG alpha=2 n=3,
  porosity 0.4, Sres 0.1, Ssat 1, Ss 1e-4, hydrostatic IC with the water table
  at z = 2 m, top flux -0.05 m/h, no-flow sides, constant head at the bottom,
  10 steps of 0.1 h.
* ``hetero`` (config 2): 512x512x50 heterogeneous box, sigma_lnK 1.5,
  correlation 32x32x4 cells, alpha perturbed +-20 % per cell (per-cell VG
  files), 20 steps of 0.05 h.
* ``ensemble_member`` / ``ensemble`` (config 3): 48 members of uneven size,
  per member nx = ny from {64, 96, 128, 192}, nz from {16, 24, 32, 40},
  sigma_lnK ~ U[0.5, 2], alpha ~ U[0.5, 4], n ~ U[1.4, 3], top flux ~
  U[-0.1, -0.02] m/h, config-0 physics otherwise, 10 steps of 0.1 h.
* ``overland`` (config 1): 256x256x20 hillslope, dx = dy = 10 m, dz = 0.2 m,
  terrain-following grid with smoothed random slopes |S| in [1e-4, 5e-2],
  Manning's n 5.5e-5, kinematic overland flow on the top face with rain
  0.01 m/h for 2 h then none until 4 h, two layers (K 0.1 / 0.005 m/h,
  alpha 3.5 / 1.0, n 2.0 / 1.8), water table 1 m below the surface,
  16 steps of 0.25 h.
* ``adjoint_box`` (config 4): 128x128x32 with config-0 physics, 20 steps.

Every size can be scaled down (``nx``, ``ny``, ``nz`` overrides) for parity
tests; fields stay seeded.
"""

from __future__ import annotations

import numpy as np

from .problem import BC, BC_DIRICHLET, BC_FLUX, BC_OVERLAND_KIN, RichardsProblem, SolverSettings
from .synth import lognormal_field, smoothed_slopes


def box(nx=64, ny=64, nz=32, nsteps=10, dt=0.1, seed=0, sigma=1.0, corr=8.0,
        solver: SolverSettings = None) -> RichardsProblem:
    lnk = lognormal_field((nz, ny, nx), (corr, corr, corr), seed, sigma=sigma)
    perm = 0.01 * np.exp(lnk)
    p = RichardsProblem(nx=nx, ny=ny, nz=nz, dx=1.0, dy=1.0, dz=0.5, perm=perm,
                        porosity=0.4, specific_storage=1e-4, vg_alpha=2.0, vg_n=3.0,
                        s_res=0.1, s_sat=1.0, dt=dt, nsteps=nsteps,
                        solver=solver or SolverSettings(), name="box")
    p.bc = {
        "x_lower": BC(BC_FLUX, (0.0,)),
        "x_upper": BC(BC_FLUX, (0.0,)),
        "y_lower": BC(BC_FLUX, (0.0,)),
        "y_upper": BC(BC_FLUX, (0.0,)),
        "z_lower": BC(BC_DIRICHLET, (2.0,), ref_patch="z_lower"),
        "z_upper": BC(BC_FLUX, (-0.05,)),
    }
    p.ic = p.hydrostatic_ic(2.0, "z_lower")
    return p


def hetero(nx=512, ny=512, nz=50, nsteps=20, dt=0.05, seed=2,
           solver: SolverSettings = None) -> RichardsProblem:
    lnk = lognormal_field((nz, ny, nx), (4.0, 32.0, 32.0), seed, sigma=1.5)
    perm = 0.01 * np.exp(lnk)
    rng = np.random.default_rng(seed + 1000)
    alpha = 2.0 * (1.0 + 0.4 * (rng.random((nz, ny, nx)) - 0.5))
    p = RichardsProblem(nx=nx, ny=ny, nz=nz, dx=1.0, dy=1.0, dz=0.5, perm=perm,
                        porosity=0.4, specific_storage=1e-4, vg_alpha=alpha,
                        vg_n=np.full((nz, ny, nx), 3.0), s_res=0.1, s_sat=1.0,
                        dt=dt, nsteps=nsteps, solver=solver or SolverSettings(),
                        name="hetero")
    p.bc = {
        "x_lower": BC(BC_FLUX, (0.0,)),
        "x_upper": BC(BC_FLUX, (0.0,)),
        "y_lower": BC(BC_FLUX, (0.0,)),
        "y_upper": BC(BC_FLUX, (0.0,)),
        "z_lower": BC(BC_DIRICHLET, (2.0,), ref_patch="z_lower"),
        "z_upper": BC(BC_FLUX, (-0.05,)),
    }
    p.ic = p.hydrostatic_ic(2.0, "z_lower")
    return p


def overland(nx=256, ny=256, nz=20, nsteps=16, dt=0.25, seed=1, wt_depth=1.0,
             mannings=5.5e-5, rain=-0.01, rain_steps=8, dry_steps=8,
             solver: SolverSettings = None, kind: int = BC_OVERLAND_KIN) -> RichardsProblem:
    """Config 1.  ``wt_depth`` is the water-table depth below the surface
    (negative: ponded start); ``kind`` the overland routing of the top face:
    BC_OVERLAND_KIN (OverlandKinematic), BC_OVERLAND (OverlandFlow) or
    BC_OVERLAND_DIFF (OverlandDiffusive)."""
    shape = (nz, ny, nx)
    top = np.arange(nz)[:, None, None] >= nz // 2
    perm = np.where(top, 0.1, 0.005) * np.ones(shape)
    alpha = np.where(top, 3.5, 1.0) * np.ones(shape)
    vg_n = np.where(top, 2.0, 1.8) * np.ones(shape)
    p = RichardsProblem(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=0.2, perm=perm,
                        porosity=0.4, specific_storage=1e-4, vg_alpha=alpha, vg_n=vg_n,
                        s_res=0.1, s_sat=1.0, dt=dt, nsteps=nsteps,
                        solver=solver or SolverSettings(), name="overland")
    p.terrain_following = True
    p.slope_x = smoothed_slopes((ny, nx), seed, 1e-4, 5e-2)
    p.slope_y = smoothed_slopes((ny, nx), seed + 1, 1e-4, 5e-2)
    p.mannings = mannings
    p.bc = {face: BC(BC_FLUX, (0.0,)) for face in
            ("x_lower", "x_upper", "y_lower", "y_upper", "z_lower")}
    p.bc["z_upper"] = BC(kind, (rain, 0.0), lengths=(rain_steps, dry_steps))
    p.ic = p.hydrostatic_ic(-wt_depth, "z_upper")
    return p


ENSEMBLE_NXY = (64, 96, 128, 192)
ENSEMBLE_NZ = (16, 24, 32, 40)


def ensemble_member(m: int, seed: int = 3, nxy=ENSEMBLE_NXY, nz=ENSEMBLE_NZ,
                    nsteps: int = 10, solver: SolverSettings = None) -> RichardsProblem:
    """Member m of the ensemble: size and parameters drawn from its own seeded
    stream (``nxy`` / ``nz`` choose the size sets, smaller ones for tests)."""
    rng = np.random.default_rng(seed * 100003 + m)
    n_xy = int(rng.choice(np.asarray(nxy)))
    n_z = int(rng.choice(np.asarray(nz)))
    sigma = float(rng.uniform(0.5, 2.0))
    alpha = float(rng.uniform(0.5, 4.0))
    vg_n = float(rng.uniform(1.4, 3.0))
    top = float(rng.uniform(-0.1, -0.02))
    p = box(nx=n_xy, ny=n_xy, nz=n_z, nsteps=nsteps, dt=0.1, seed=seed * 1009 + m,
            sigma=sigma, solver=solver)
    p.vg_alpha = alpha
    p.vg_n = vg_n
    p.bc["z_upper"] = BC(BC_FLUX, (top,))
    p.name = f"member{m}"
    return p


def ensemble(n: int = 48, seed: int = 3, **kw):
    return [ensemble_member(m, seed=seed, **kw) for m in range(n)]


def adjoint_box(nx=128, ny=128, nz=32, nsteps=20, seed=4) -> RichardsProblem:
    return box(nx=nx, ny=ny, nz=nz, nsteps=nsteps, dt=0.1, seed=seed)


__all__ = ["box", "hetero", "overland", "ensemble_member", "ensemble", "adjoint_box"]
