"""PyTorch autograd over the discrete adjoint of the implicit Richards steps.

This is the Python-side face of pfgpu_adjoint_record / pfgpu_adjoint_gradient
(the pftools layer of ParFlow has no adjoint; the forward model it wraps is
the KINSOL timestep of pfsimulator/parflow_lib/solver_richards.c:2965-3406).

``RichardsObservation`` maps per-cell parameter fields (ln K, van Genuchten
alpha and n, each (nz, ny, nx) float64) to the simulated pressure heads at a
fixed set of observation cells and steps: a tensor of shape
(len(obs_steps), len(obs_cells)).  Any differentiable loss built on that
tensor back-propagates through the adjoint.

The C ABI evaluates the adjoint of one objective, g = sum (p_n[c] - obs)^2,
whose gradient with respect to the observed pressures is 2 (p - obs).  For an
upstream gradient w the wrapper passes obs = p - s w / 2, so dg/dp = s w, and
divides the returned parameter gradients by s.  The adjoint is linear in
dg/dp, so this is the exact vector-Jacobian product of the observation map;
s scales s w to the size of p so that forming p - obs loses no digits of w.

Every forward solve records the trajectory on the GPU handle; a backward pass
whose forward is no longer the handle's latest recorded trajectory solves the
forward again first (from the fields saved for backward).
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .problem import RichardsProblem
from .solver import RichardsGPU


class RichardsAdjointModel:
    """A Richards problem on one GPU handle with a fixed observation design.

    prob       -- the problem (grid, physics, constant boundary conditions,
                  time plan); its permeability and van Genuchten fields are
                  replaced by the tensors passed to each forward call.
    obs_steps  -- 1-based step numbers whose pressures are observed.
    obs_cells  -- dense interior cell indices i + nx*(j + ny*k).
    tol        -- relative residual of the transposed-Jacobian GMRES solves.

    The handle is FP64: the mixed forms store the Jacobian in FP32, which the
    adjoint's transposed solves must not see.
    """

    def __init__(self, prob: RichardsProblem, obs_steps: Sequence[int],
                 obs_cells: Sequence[int], device: int = 0, tol: float = 1e-10):
        self.prob = prob
        self.obs_steps = np.ascontiguousarray(obs_steps, dtype=np.int32)
        self.obs_cells = np.ascontiguousarray(obs_cells, dtype=np.int64)
        self.nsteps = int(self.obs_steps.max())
        if self.obs_steps.min() < 1 or self.nsteps > len(prob.time_plan()):
            raise ValueError("observation steps must lie in 1..number of timesteps")
        if self.obs_cells.min() < 0 or self.obs_cells.max() >= prob.nx * prob.ny * prob.nz:
            raise ValueError("observation cell index out of range")
        self.tol = tol
        # per-cell van Genuchten fields from the start, so the handle keeps
        # per-cell arrays for every forward call
        shape = prob.shape
        if np.isscalar(prob.vg_alpha):
            prob.vg_alpha = np.full(shape, float(prob.vg_alpha))
        if np.isscalar(prob.vg_n):
            prob.vg_n = np.full(shape, float(prob.vg_n))
        self.gpu = RichardsGPU(prob, precision="fp64", device=device)
        self._recorded = None       # token of the forward held on the handle
        self._tokens = 0

    def close(self):
        self.gpu.close()

    def forward(self, lnk: np.ndarray, alpha: np.ndarray, vg_n: np.ndarray):
        """Solve the time plan with these fields, record the trajectory and
        return (observed pressures, token of this trajectory)."""
        p = self.prob
        p.perm = np.exp(np.asarray(lnk, dtype=np.float64).reshape(p.shape))
        p.vg_alpha = np.asarray(alpha, dtype=np.float64).reshape(p.shape)
        p.vg_n = np.asarray(vg_n, dtype=np.float64).reshape(p.shape)
        g = self.gpu
        g.update_fields()
        g.set_pressure(p.initial_pressure())
        g.adjoint_record(self.nsteps)
        out = np.empty((len(self.obs_steps), len(self.obs_cells)))
        want = {int(s): k for k, s in enumerate(self.obs_steps)}
        for n, (t, dt) in enumerate(p.time_plan()[:self.nsteps], start=1):
            g.set_time(t)
            g.advance(1, dt)
            if n in want:
                out[want[n]] = g.get_pressure().ravel()[self.obs_cells]
        self._tokens += 1
        self._recorded = self._tokens
        return out, self._recorded

    def vjp(self, p_obs: np.ndarray, w: np.ndarray):
        """Vector-Jacobian product of the observation map at the recorded
        trajectory: returns (w^T dp/d lnK, w^T dp/d alpha, w^T dp/d n)."""
        w = np.asarray(w, dtype=np.float64).reshape(p_obs.shape)
        wmax = float(np.abs(w).max()) if w.size else 0.0
        shape = self.prob.shape
        if wmax == 0.0:
            return tuple(np.zeros(shape) for _ in range(3))
        s = max(1.0, float(np.abs(p_obs).max())) / wmax
        obs = p_obs - 0.5 * s * w
        _, g_lnk, g_a, g_n = self.gpu.adjoint_gradient(self.obs_steps, self.obs_cells, obs,
                                                       tol=self.tol)
        return g_lnk / s, g_a / s, g_n / s


def _torch():
    import torch

    return torch


def _make_function():
    torch = _torch()

    class RichardsObservation(torch.autograd.Function):
        """(lnK, alpha, n) -> observed pressures, differentiable by the
        discrete adjoint.  Call through :func:`observe`."""

        @staticmethod
        def forward(ctx, lnk, alpha, vg_n, model: RichardsAdjointModel):
            arrs = [t.detach().to("cpu", torch.float64).numpy() for t in (lnk, alpha, vg_n)]
            p_obs, token = model.forward(*arrs)
            ctx.model = model
            ctx.token = token
            ctx.p_obs = p_obs
            ctx.save_for_backward(lnk, alpha, vg_n)
            return torch.from_numpy(p_obs).to(lnk.device)

        @staticmethod
        def backward(ctx, grad_out):
            model = ctx.model
            lnk, alpha, vg_n = ctx.saved_tensors
            if model._recorded != ctx.token:
                # the handle holds a later trajectory: solve this forward again
                arrs = [t.detach().to("cpu", torch.float64).numpy() for t in (lnk, alpha, vg_n)]
                _, ctx.token = model.forward(*arrs)
            w = grad_out.detach().to("cpu", torch.float64).numpy()
            g = model.vjp(ctx.p_obs, w)
            outs = [torch.from_numpy(np.ascontiguousarray(a)).to(t.device, t.dtype)
                    if need else None
                    for a, t, need in zip(g, (lnk, alpha, vg_n), ctx.needs_input_grad[:3])]
            return outs[0], outs[1], outs[2], None

    return RichardsObservation


_FUNCTION = None


def observe(lnk, alpha, vg_n, model: RichardsAdjointModel):
    """Simulated pressure heads at the model's observation steps and cells,
    shape (len(obs_steps), len(obs_cells)), differentiable with respect to the
    per-cell fields lnk, alpha and vg_n (float64 tensors of shape (nz, ny, nx))."""
    global _FUNCTION
    if _FUNCTION is None:
        _FUNCTION = _make_function()
    return _FUNCTION.apply(lnk, alpha, vg_n, model)


def misfit(lnk, alpha, vg_n, model: RichardsAdjointModel, obs_values,
           sigma: Optional[float] = None):
    """Sum of squared differences between simulated and observed heads
    (divided by sigma^2 when given), differentiable by the adjoint."""
    torch = _torch()
    sim = observe(lnk, alpha, vg_n, model)
    r = sim - torch.as_tensor(obs_values, dtype=sim.dtype, device=sim.device)
    out = (r * r).sum()
    return out if sigma is None else out / (sigma * sigma)


__all__ = ["RichardsAdjointModel", "observe", "misfit"]
