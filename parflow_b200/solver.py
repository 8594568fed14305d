"""Host-side mirror of ParFlow's Richards nonlinear-solver interface over the
C ABI of libpfgpu.

:class:`RichardsGPU` plays the role of the PFModules on this path, with the
same argument meaning: ``nl_function_eval`` (NlFunctionEval,
pfsimulator/parflow_lib/nl_function_eval.c:167), ``jacobian_matvec``
(KINSolMatVec, richards_jacobian_eval.c:165), ``pc_setup`` / ``pc_apply``
(KinsolPC, kinsol_pc.c:58-149), ``saturation`` (Saturation,
problem_saturation.c:108), ``newton_solve`` (KinsolNonlinSolver,
kinsol_nonlin_solver.c:297, returning nonzero when KINSOL fails so the caller
halves dt) and ``advance`` (the AdvanceRichards step body,
solver_richards.c:2965-3406).

Arrays are accepted as numpy arrays of shape (nz, ny, nx) (interior cells;
converted to ParFlow's ghost-framed layout at the boundary) or as torch CUDA
tensors already in the ghost-framed layout (passed by device pointer, no copy).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import lib as L
from .problem import FACES, RichardsProblem

_ETA = {"EtaConstant": 0, "Walker1": 1, "Walker2": 2}


def pad(a: np.ndarray) -> np.ndarray:
    """(nz, ny, nx) interior -> (nz+2, ny+2, nx+2) ParFlow Subvector layout."""
    a = np.asarray(a, dtype=np.float64)
    out = np.zeros((a.shape[0] + 2, a.shape[1] + 2, a.shape[2] + 2))
    out[1:-1, 1:-1, 1:-1] = a
    return out


def unpad(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a[1:-1, 1:-1, 1:-1])


def _ptr(a):
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


class RichardsGPU:
    """One Richards problem resident on a GPU."""

    def __init__(self, prob: RichardsProblem, precision: str = "fp64", device: int = 0):
        self.prob = prob
        self.lib = L.load()
        s = prob.solver
        d = L.Desc()
        d.abi_version = L.ABI_VERSION
        d.nx, d.ny, d.nz = prob.nx, prob.ny, prob.nz
        d.dx, d.dy, d.dz = prob.dx, prob.dy, prob.dz
        d.gravity, d.viscosity, d.density = prob.gravity, prob.viscosity, prob.density
        d.porosity, d.specific_storage = prob.porosity, prob.specific_storage
        file_mode = prob.vg_from_file()
        d.vg_alpha = float(prob.field3d(prob.vg_alpha).flat[0])
        d.vg_n = float(prob.field3d(prob.vg_n).flat[0])
        d.s_res = float(prob.field3d(prob.s_res).flat[0])
        d.s_sat = float(prob.field3d(prob.s_sat).flat[0])
        d.vg_from_file = 1 if file_mode else 0
        self._zm = np.ascontiguousarray(prob.zmult())
        d.z_mult = self._zm.ctypes.data_as(C.POINTER(C.c_double))
        precisions = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED, "mixed16": L.PREC_MIXED_H16}
        if precision not in precisions:
            raise ValueError(f"precision must be one of {sorted(precisions)}")
        d.precision = precisions[precision]
        d.residual_tol, d.step_tol = s.residual_tol, s.step_tol
        d.max_iter, d.krylov_dim, d.max_restarts = s.max_iter, s.krylov_dim, s.max_restarts
        d.eta_choice = _ETA[s.eta_choice]
        d.eta_value, d.eta_alpha, d.eta_gamma = s.eta_value, s.eta_alpha, s.eta_gamma
        d.mg_max_levels = s.mg_max_levels
        for q in range(3):
            d.mg_max_min_n[q] = s.mg_max_min_n[q]
        d.mg_smoother = s.smoother_code()
        d.wjacobi_weight = s.smoother_weight()
        self.desc = d
        self.precision = precision
        h = self.lib.pfgpu_create(C.byref(d), device)
        if not h:
            raise L.PfgpuError("pfgpu_create failed: " + L.last_error())
        self.h = C.c_void_p(h)
        # descriptor scalars of the van Genuchten fields, and the fields that
        # currently have a per-cell array on the device
        self._vg_scalar = {L.FIELD_VG_ALPHA: d.vg_alpha, L.FIELD_VG_N: d.vg_n,
                           L.FIELD_S_RES: d.s_res, L.FIELD_S_SAT: d.s_sat}
        self._vg_cells = set()
        if not s.use_jacobian:
            L.check(self.lib.pfgpu_set_jacobian_mode(self.h, 0, s.derivative_epsilon),
                    "set_jacobian_mode")
        if s.globalization_code() != 0:
            L.check(self.lib.pfgpu_set_globalization(self.h, s.globalization_code()),
                    "set_globalization")
        if s.pc_matrix_code():
            L.check(self.lib.pfgpu_set_pc_matrix(self.h, s.pc_matrix_code()), "set_pc_matrix")
        if prob.overland_spinup or prob.spinup_damp != (0.0, 0.0):
            L.check(self.lib.pfgpu_set_overland_spinup(self.h, int(prob.overland_spinup),
                                                       float(prob.spinup_damp[0]),
                                                       float(prob.spinup_damp[1])),
                    "set_overland_spinup")
        if s.mg_max_iter != 1:
            L.check(self.lib.pfgpu_set_mg_max_iter(self.h, s.mg_max_iter), "set_mg_max_iter")
        if prob.kr_table:
            method = {"Spline": 1, "Linear": 2}[prob.kr_table[0]]
            L.check(self.lib.pfgpu_set_relperm_table(self.h, method, int(prob.kr_table[1]),
                                                     float(prob.kr_table[2])),
                    "set_relperm_table")
        self._upload_fields()
        if prob.evap_trans is not None:
            self.set_evap_trans(prob.field3d(prob.evap_trans))
        for fid, v in ((L.FIELD_FB_X, prob.fbx), (L.FIELD_FB_Y, prob.fby), (L.FIELD_FB_Z, prob.fbz)):
            if v is not None:
                L.check(self.lib.pfgpu_set_field(self.h, fid, _ptr(pad(prob.field3d(v)))),
                        "set_field (flow barrier)")
        self.set_time(prob.start_time + prob.dt)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pfgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- setup ---------------------------------------------------------------
    def _upload_fields(self):
        p = self.prob
        if p.terrain_following or any(bc.kind in (L.BC_OVERLAND_KIN, L.BC_OVERLAND_DIFF, L.BC_OVERLAND)
                                        for bc in p.bc.values()):
            self._upload_surface()
        L.check(self.lib.pfgpu_set_field(self.h, L.FIELD_PERM_X, _ptr(pad(p.field3d(p.perm)))),
                "set_field perm")
        if p.vg_from_file():
            for fid, v in ((L.FIELD_VG_ALPHA, p.vg_alpha), (L.FIELD_VG_N, p.vg_n),
                           (L.FIELD_S_RES, p.s_res), (L.FIELD_S_SAT, p.s_sat)):
                a = p.field3d(v)
                if np.all(a == a.flat[0]) and a.flat[0] == self._vg_scalar[fid]:
                    # the descriptor scalar serves every cell; drop a per-cell
                    # array left by an earlier upload
                    if fid in self._vg_cells:
                        L.check(self.lib.pfgpu_set_field(self.h, fid, None), "clear field vg")
                        self._vg_cells.discard(fid)
                    continue
                L.check(self.lib.pfgpu_set_field(self.h, fid, _ptr(pad(a))), "set_field vg")
                self._vg_cells.add(fid)

    # ---- PFB files of the device state ------------------------------------------
    _PFB = {"pressure": L.PFB_PRESSURE, "saturation": L.PFB_SATURATION,
            "perm_x": L.FIELD_PERM_X, "perm_y": L.FIELD_PERM_Y, "perm_z": L.FIELD_PERM_Z,
            "vg_alpha": L.FIELD_VG_ALPHA, "vg_n": L.FIELD_VG_N, "s_res": L.FIELD_S_RES,
            "s_sat": L.FIELD_S_SAT}

    def write_pfb(self, path: str, what: str = "pressure", origin=(0.0, 0.0, 0.0)):
        """WritePFBinary of the device pressure or of the saturation at it."""
        L.check(self.lib.pfgpu_write_pfb(self.h, self._PFB[what], os.fsencode(path),
                                         *[float(v) for v in origin]), "write_pfb")

    def read_pfb(self, path: str, what: str = "pressure"):
        """ReadPFBinary into the device pressure or a cell field."""
        L.check(self.lib.pfgpu_read_pfb(self.h, self._PFB[what], os.fsencode(path)), "read_pfb")
        if what in ("vg_alpha", "vg_n", "s_res", "s_sat"):
            self._vg_cells.add(self._PFB[what])

    def update_fields(self):
        """Re-upload the problem's cell fields (permeability, van Genuchten,
        surface) after they changed, e.g. between runs of a parameter study."""
        self._upload_fields()

    def _upload_surface(self):
        """Slopes and Manning's n in ParFlow's 2-D layout (pfgpu_set_surface)."""
        p = self.prob
        pad2 = lambda a: np.pad(np.asarray(a, dtype=np.float64), 1)
        self._surf = [pad2(p.field2d(p.slope_x)), pad2(p.field2d(p.slope_y)),
                      pad2(p.field2d(p.mannings))]
        L.check(self.lib.pfgpu_set_surface(self.h, *[_ptr(a) for a in self._surf],
                                           1 if p.terrain_following else 0, 1.0e-5),
                "set_surface")

    def set_time(self, t: float):
        """Upload the boundary tables BCPressure would build at time t."""
        self.t = t
        for f, (typ, vals) in enumerate(self.prob.bc_values(t)):
            v = np.ascontiguousarray(vals, dtype=np.float64)
            L.check(self.lib.pfgpu_set_bc(self.h, f, typ, _ptr(v)), f"set_bc {FACES[f]}")

    # ---- function-level operators (ParFlow layout in/out) -------------------
    def _io(self, a):
        return a if hasattr(a, "data_ptr") else pad(a)

    def solve_graph(self, mode: int = -1) -> int:
        """Newton solves as one CUDA graph launch (mode 1, the default) or
        host-driven (0); mode -1 returns 1 if the last solve ran as a graph."""
        r = self.lib.pfgpu_solve_graph(self.h, int(mode))
        if mode == -1:
            return int(r)
        L.check(r, "solve_graph")
        return 0

    def set_evap_trans(self, et):
        """Per-cell land-surface sink/source [1/h] (interior (nz, ny, nx)), or
        None to clear it."""
        if et is None:
            L.check(self.lib.pfgpu_set_evap_trans(self.h, None), "set_evap_trans")
            return
        a = pad(np.broadcast_to(np.asarray(et, dtype=np.float64), self.prob.shape))
        L.check(self.lib.pfgpu_set_evap_trans(self.h, _ptr(a)), "set_evap_trans")

    def face_velocities(self, dt, p=None, p_old=None, s_old=None):
        """Face velocities and overland fluxes of the residual at p (None:
        the handle's pressure state and the last step's old state), dense:
        vx (nz, ny, nx+1), vy (nz, ny+1, nx), vz (nz+1, ny, nx), qx, qy
        (ny, nx)."""
        nz, ny, nx = self.prob.shape
        vx = np.zeros((nz + 2, ny + 2, nx + 3))
        vy = np.zeros((nz + 2, ny + 3, nx + 2))
        vz = np.zeros((nz + 5, ny + 4, nx + 4))  # two ghost layers, as ParFlow's z_velocity
        qx = np.zeros((3, ny + 2, nx + 2))
        qy = np.zeros((3, ny + 2, nx + 2))
        bufs = []  # padded inputs, alive through the call
        for a in (p, p_old, s_old):
            bufs.append(None if a is None else pad(np.ascontiguousarray(a, dtype=np.float64)))
        rc = self.lib.pfgpu_face_velocities(self.h, *[None if b is None else _ptr(b) for b in bufs],
                                            float(dt), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(qx),
                                            _ptr(qy))
        L.check(rc, "face_velocities")
        return (unpad(vx), unpad(vy), np.ascontiguousarray(vz[2:-2, 2:-2, 2:-2]),
                np.ascontiguousarray(qx[1, 1:-1, 1:-1]),
                np.ascontiguousarray(qy[1, 1:-1, 1:-1]))

    def nl_function_eval(self, p, p_old, s_old, dt):
        f = np.zeros(tuple(x + 2 for x in self.prob.shape))
        L.check(self.lib.pfgpu_nl_function_eval(self.h, _ptr(self._io(p)), _ptr(self._io(p_old)),
                                                _ptr(self._io(s_old)), dt, _ptr(f)),
                "nl_function_eval")
        return unpad(f)

    def saturation(self, p):
        s = np.zeros(tuple(x + 2 for x in self.prob.shape))
        L.check(self.lib.pfgpu_saturation(self.h, _ptr(self._io(p)), _ptr(s)), "saturation")
        return unpad(s)

    def set_old_pressure(self, p_old):
        """The step's old pressure, read by the Jacobian's diffusive overland
        terms (RichardsJacobianEval's old_pressure argument)."""
        L.check(self.lib.pfgpu_set_old_pressure(self.h, _ptr(self._io(p_old))), "set_old_pressure")

    def jacobian_matvec(self, p, dt, x, p_old=None):
        if p_old is not None:
            self.set_old_pressure(p_old)
        y = np.zeros(tuple(n + 2 for n in self.prob.shape))
        L.check(self.lib.pfgpu_jacobian_matvec(self.h, _ptr(self._io(p)), dt, _ptr(self._io(x)),
                                               _ptr(y)), "jacobian_matvec")
        return unpad(y)

    def pc_setup(self, p, dt, p_old=None):
        if p_old is not None:
            self.set_old_pressure(p_old)
        L.check(self.lib.pfgpu_pc_setup(self.h, _ptr(self._io(p)), dt), "pc_setup")

    def pc_apply(self, r):
        z = np.zeros(tuple(n + 2 for n in self.prob.shape))
        L.check(self.lib.pfgpu_pc_apply(self.h, _ptr(self._io(r)), _ptr(z)), "pc_apply")
        return unpad(z)

    def mg_levels(self):
        n = C.c_int()
        dims = (C.c_int * 512)()
        L.check(self.lib.pfgpu_mg_levels(self.h, C.byref(n), dims, 128), "mg_levels")
        return [tuple(dims[4 * l: 4 * l + 4]) for l in range(n.value)]

    def newton_solve(self, p_init, p_old, s_old, dt):
        """KinsolNonlinSolver: returns (p, status, stats); status 0 = converged."""
        p = pad(p_init)
        st = L.Stats()
        rc = L.check(self.lib.pfgpu_newton_solve(self.h, _ptr(self._io(p_old)),
                                                 _ptr(self._io(s_old)), dt, _ptr(p),
                                                 C.byref(st)), "newton_solve")
        return unpad(p), rc, st

    def newton_solve_sat(self, p_init, p_old, s_old, dt):
        """newton_solve and the saturation at the solution in one call:
        returns (p, s, status)."""
        p = pad(p_init)
        sat = np.zeros_like(p)
        st = L.Stats()
        rc = L.check(self.lib.pfgpu_newton_solve_sat(self.h, _ptr(self._io(p_old)),
                                                     _ptr(self._io(s_old)), dt, _ptr(p),
                                                     _ptr(sat), C.byref(st)), "newton_solve_sat")
        return unpad(p), unpad(sat), rc

    # ---- device-resident stepping ---------------------------------------------
    def set_pressure(self, p):
        L.check(self.lib.pfgpu_set_pressure(self.h, _ptr(self._io(p))), "set_pressure")

    def get_pressure(self, out=None):
        if out is not None and hasattr(out, "data_ptr"):
            L.check(self.lib.pfgpu_get_pressure(self.h, _ptr(out)), "get_pressure")
            return out
        p = np.zeros(tuple(n + 2 for n in self.prob.shape))
        L.check(self.lib.pfgpu_get_pressure(self.h, _ptr(p)), "get_pressure")
        return unpad(p)

    def advance(self, nsteps: int = 1, dt: Optional[float] = None):
        """Advance the device state nsteps steps; returns per-step stats."""
        dt = self.prob.dt if dt is None else dt
        stats = (L.Stats * max(1, nsteps))()
        rc = L.check(self.lib.pfgpu_advance(self.h, dt, nsteps, stats), "advance")
        if rc != L.OK:
            raise L.PfgpuError("advance: " + L.last_error())
        return [stats[i] for i in range(nsteps)]

    def run(self, nsteps: Optional[int] = None):
        """Solve the problem's time loop step by step (BCs re-evaluated per
        step); returns (pressures after each step, stats per step)."""
        prob = self.prob
        plan = prob.time_plan()
        nsteps = len(plan) if nsteps is None else nsteps
        self.set_pressure(prob.initial_pressure())
        ps, sts = [], []
        for t, dt in plan[:nsteps]:
            self.set_time(t)
            sts.extend(self.advance(1, dt))
            ps.append(self.get_pressure())
        return ps, sts

    def upload_bc_cycles(self):
        """Every face's time cycle as device tables (pfgpu_set_bc_cycle): one
        face table per interval, selected by the native time loop."""
        p = self.prob
        base = p.base_unit if p.base_unit is not None else p.dt
        for f, face in enumerate(FACES):
            bc = p.bc.get(face)
            kind = bc.kind if bc is not None else L.BC_FLUX
            values = tuple(bc.values) if bc is not None else (0.0,)
            lengths = tuple(bc.lengths) if bc is not None else (1,)
            repeat = bc.repeat if bc is not None else -1
            tables = []
            for v in values:
                if kind == L.BC_DIRICHLET:
                    tables.append(p._dir_equil_values(face, float(v), bc.ref_patch))
                else:
                    tables.append(np.full(p.face_shape(face), float(v)))
            vals = np.ascontiguousarray(np.stack(tables), dtype=np.float64)
            n = len(values)
            types = (C.c_int * n)(*([kind] * n))
            lens = (C.c_int * n)(*[int(x) for x in lengths])
            L.check(self.lib.pfgpu_set_bc_cycle(
                self.h, f, n, types, vals.ctypes.data_as(C.POINTER(C.c_double)), lens,
                int(repeat), float(base), float(p.start_time)), f"set_bc_cycle {face}")

    def run_device(self, max_steps: Optional[int] = None, dump_interval: Optional[float] = None,
                   growth=None):
        """The problem's time loop as one native call (pfgpu_run): time-cycled
        boundary tables on the device, SelectTimeStep (constant dt, or
        growth = (initial, factor, min, max)), dump-time snapping, the dt-halving
        retry.  Returns (final pressure, times, dts, stats per step)."""
        p = self.prob
        self.upload_bc_cycles()
        fails = int(p.solver.max_convergence_failures)
        if growth is None:
            L.check(self.lib.pfgpu_set_time_step(self.h, 0, float(p.dt), 1.0, 0.0, 0.0, fails),
                    "set_time_step")
        else:
            init, factor, lo, hi = (float(v) for v in growth)
            L.check(self.lib.pfgpu_set_time_step(self.h, 1, init, factor, lo, hi, fails),
                    "set_time_step")
        n_max = max_steps if max_steps is not None else 10 * p.nsteps + 10
        times = (C.c_double * n_max)()
        dts = (C.c_double * n_max)()
        stats = (L.Stats * n_max)()
        n = C.c_int()
        dump = float(p.dt) if dump_interval is None else float(dump_interval)
        self.set_pressure(p.initial_pressure())
        rc = L.check(self.lib.pfgpu_run(self.h, float(p.start_time), float(p.stop_time()), dump,
                                        n_max, times, dts, stats, C.byref(n)), "run")
        if rc != L.OK:
            raise L.PfgpuError("run: " + L.last_error())
        k = n.value
        return (self.get_pressure(), list(times[:k]), list(dts[:k]), [stats[i] for i in range(k)])

    # ---- discrete adjoint ------------------------------------------------------
    def adjoint_record(self, max_steps: int):
        """Start recording the trajectory at the current pressure."""
        L.check(self.lib.pfgpu_adjoint_record(self.h, max_steps), "adjoint_record")

    def adjoint_gradient(self, obs_steps, obs_cells, obs_values, tol: float = 1e-10):
        """Misfit sum (p_n[c] - obs)^2 over the observed steps/cells of the
        recorded trajectory and its gradient w.r.t. per-cell ln K, alpha, n
        (each (nz, ny, nx)).  obs_cells are dense indices i + nx*(j + ny*k);
        obs_values has shape (len(obs_steps), len(obs_cells))."""
        steps = np.ascontiguousarray(obs_steps, dtype=np.int32)
        cells = np.ascontiguousarray(obs_cells, dtype=np.int64)
        vals = np.ascontiguousarray(obs_values, dtype=np.float64).reshape(len(steps), len(cells))
        shape_p = tuple(n + 2 for n in self.prob.shape)
        g = [np.zeros(shape_p) for _ in range(3)]
        misfit = C.c_double()
        rc = self.lib.pfgpu_adjoint_gradient(
            self.h, len(steps), steps.ctypes.data_as(C.POINTER(C.c_int)), len(cells),
            cells.ctypes.data_as(C.POINTER(C.c_longlong)),
            vals.ctypes.data_as(C.POINTER(C.c_double)), tol, C.byref(misfit),
            *[_ptr(a) for a in g])
        L.check(rc, "adjoint_gradient")
        if rc != L.OK:
            raise L.PfgpuError("adjoint_gradient: " + L.last_error())
        return misfit.value, unpad(g[0]), unpad(g[1]), unpad(g[2])

    def time_kernel(self, name: str, reps: int = 10):
        """(ms per launch, algorithmic bytes per launch) of one library kernel."""
        ms, by = C.c_double(), C.c_double()
        L.check(self.lib.pfgpu_time_kernel(self.h, L.KERNELS[name], reps, C.byref(ms), C.byref(by)),
                "time_kernel")
        return ms.value, by.value

    def autotune(self, reps: int = 10) -> dict:
        """Pick the thread-block shapes of the residual, Jacobian and matvec
        launches for this grid (pfgpu_autotune); returns them, (0, 0) being
        the built-in heuristic."""
        out = (C.c_int * 6)()
        L.check(self.lib.pfgpu_autotune(self.h, reps, out), "autotune")
        return {"residual": (out[0], out[1]), "jacobian": (out[2], out[3]),
                "matvec": (out[4], out[5])}

    def kernel_launches(self) -> int:
        return int(self.lib.pfgpu_kernel_launches(self.h))

    def stream(self) -> int:
        return int(self.lib.pfgpu_stream(self.h) or 0)


__all__ = ["RichardsGPU", "pad", "unpad"]


def ensemble_advance(members, nsteps: int = 1, dts=None, threads: int = 0):
    """Advance several :class:`RichardsGPU` problems concurrently by nsteps
    steps each (pfgpu_ensemble_advance): every member on its own stream,
    ``threads`` host threads driving their Newton loops (0 = one per member).
    Boundary tables and pressures must already be set.  Returns the per-member
    lists of per-step stats; raises on an error or a step that fails."""
    n = len(members)
    if n == 0:
        return []
    lib = members[0].lib
    dts = [m.prob.dt for m in members] if dts is None else list(dts)
    handles = (C.c_void_p * n)(*[m.h.value for m in members])
    dt_arr = (C.c_double * n)(*dts)
    per = max(1, nsteps)
    stats = (L.Stats * (n * per))()
    status = (C.c_int * n)()
    rc = lib.pfgpu_ensemble_advance(handles, n, dt_arr, nsteps, threads, stats, status)
    if rc != L.OK:
        raise L.PfgpuError(f"ensemble_advance failed ({rc}): {L.last_error()}")
    return [[stats[m * per + s] for s in range(nsteps)] for m in range(n)]
