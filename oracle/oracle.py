"""Test infrastructure: ctypes binding of the CPU restatement in
oracle/pforacle.c (built as oracle/liboracle.so).  Used only by tests/, the
package smoke check and bench.py's CPU-baseline leg, as the checker.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)


class Problem(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("gravity", C.c_double), ("viscosity", C.c_double), ("density", C.c_double),
                ("kx", _dp), ("ky", _dp), ("kz", _dp),
                ("porosity", C.c_double), ("sstorage", C.c_double),
                ("alpha", _dp), ("n", _dp), ("s_res", _dp), ("s_sat", _dp),
                ("vg_from_file", C.c_int),
                ("z_mult", _dp),
                ("bc_type", C.c_int * 6),
                ("bc_val", _dp * 6),
                ("sslope_x", _dp), ("sslope_y", _dp),
                ("tslope_x", _dp), ("tslope_y", _dp),
                ("mannings", _dp),
                ("ov_epsilon", C.c_double),
                ("ov_p_old", _dp),
                ("kr_table", C.c_void_p),
                ("evap_trans", _dp), ("fbx", _dp), ("fby", _dp), ("fbz", _dp),
                ("ov_spinup", C.c_int), ("ov_damp_p1", C.c_double), ("ov_damp_p2", C.c_double)]


class FluxOut(C.Structure):
    _fields_ = [("vx", _dp), ("vy", _dp), ("vz", _dp), ("qx", _dp), ("qy", _dp)]


class Settings(C.Structure):
    _fields_ = [("residual_tol", C.c_double), ("step_tol", C.c_double),
                ("max_iter", C.c_int), ("krylov_dim", C.c_int), ("max_restarts", C.c_int),
                ("eta_choice", C.c_int),
                ("eta_value", C.c_double), ("eta_alpha", C.c_double), ("eta_gamma", C.c_double),
                ("mg_max_levels", C.c_int), ("mg_smoother", C.c_int),
                ("wjacobi_weight", C.c_double),
                ("use_jacobian", C.c_int), ("derivative_epsilon", C.c_double),
                ("globalization", C.c_int), ("mg_max_iter", C.c_int),
                ("mg_max_min_n", C.c_int * 3), ("pc_full", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("status", C.c_int), ("nni", C.c_int), ("nli", C.c_int), ("nfe", C.c_int),
                ("nps", C.c_int), ("npe", C.c_int), ("nbcf", C.c_int), ("nbktrk", C.c_int),
                ("ncfl", C.c_int), ("fnorm", C.c_double)]


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "pforacle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, src, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.pfo_residual.argtypes = [C.POINTER(Problem), C.c_double, _dp, _dp, _dp, _dp]
        L.pfo_residual_out.argtypes = [C.POINTER(Problem), C.c_double, _dp, _dp, _dp, _dp,
                                       C.POINTER(FluxOut)]
        L.pfo_jacobian.argtypes = [C.POINTER(Problem), C.c_double, _dp, C.c_int, C.POINTER(_dp)]
        L.pfo_jacobian_fd.argtypes = [C.POINTER(Problem), C.c_double, _dp, C.c_int, C.c_int,
                                      C.POINTER(_dp)]
        L.pfo_matvec7.argtypes = [C.POINTER(Problem), C.POINTER(_dp), _dp, _dp]
        L.pfo_saturation.argtypes = [C.POINTER(Problem), _dp, _dp, C.c_int]
        L.pfo_relperm.argtypes = [C.POINTER(Problem), _dp, _dp, C.c_int]
        L.pfo_mg_create.argtypes = [C.POINTER(Problem), C.POINTER(Settings)]
        L.pfo_mg_create.restype = C.c_void_p
        L.pfo_mg_setup.argtypes = [C.c_void_p, C.POINTER(_dp)]
        L.pfo_mg_setup_full.argtypes = [C.c_void_p, C.POINTER(_dp)]
        L.pfo_mg_set_wghost.argtypes = [C.c_void_p, _dp]
        L.pfo_vgtable_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.pfo_vgtable_create.restype = C.c_void_p
        L.pfo_vgtable_destroy.argtypes = [C.c_void_p]
        L.pfo_mg_apply.argtypes = [C.c_void_p, _dp, _dp]
        L.pfo_mg_num_levels.argtypes = [C.c_void_p]
        L.pfo_mg_level_info.argtypes = [C.c_void_p, C.c_int] + [C.POINTER(C.c_int)] * 4
        L.pfo_mg_destroy.argtypes = [C.c_void_p]
        L.pfo_newton_solve.argtypes = [C.POINTER(Problem), C.POINTER(Settings), C.c_double,
                                       _dp, _dp, _dp, C.POINTER(Stats)]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


ETA = {"EtaConstant": 0, "Walker1": 1, "Walker2": 2}


class Oracle:
    """Oracle view of a :class:`parflow_b200.problem.RichardsProblem`."""

    def __init__(self, prob, t: float = None):
        self.prob = prob
        self._keep = []
        nz, ny, nx = prob.shape
        k = np.ascontiguousarray(prob.field3d(prob.perm))
        a = np.ascontiguousarray(prob.field3d(prob.vg_alpha))
        n = np.ascontiguousarray(prob.field3d(prob.vg_n))
        sr = np.ascontiguousarray(prob.field3d(prob.s_res))
        ss = np.ascontiguousarray(prob.field3d(prob.s_sat))
        zm = np.ascontiguousarray(prob.zmult())
        self._keep += [k, a, n, sr, ss, zm]
        P = Problem()
        P.nx, P.ny, P.nz = nx, ny, nz
        P.dx, P.dy, P.dz = prob.dx, prob.dy, prob.dz
        P.gravity, P.viscosity, P.density = prob.gravity, prob.viscosity, prob.density
        P.kx = P.ky = P.kz = _ptr(k)
        P.porosity, P.sstorage = prob.porosity, prob.specific_storage
        P.alpha, P.n, P.s_res, P.s_sat = _ptr(a), _ptr(n), _ptr(sr), _ptr(ss)
        P.vg_from_file = 1 if prob.vg_from_file() else 0
        P.z_mult = _ptr(zm)
        # slopes and Manning's n (2-D, (ny, nx)); subsurface slopes only under
        # the terrain-following grid (solver_richards.c:562-572)
        sx = np.ascontiguousarray(prob.field2d(prob.slope_x))
        sy = np.ascontiguousarray(prob.field2d(prob.slope_y))
        man = np.ascontiguousarray(prob.field2d(prob.mannings))
        self._keep += [sx, sy, man]
        P.tslope_x, P.tslope_y, P.mannings = _ptr(sx), _ptr(sy), _ptr(man)
        if prob.terrain_following:
            P.sslope_x, P.sslope_y = _ptr(sx), _ptr(sy)
        P.ov_epsilon = 1.0e-5
        if prob.evap_trans is not None:
            et = np.ascontiguousarray(prob.field3d(prob.evap_trans), dtype=np.float64)
            self._keep.append(et)
            P.evap_trans = _ptr(et)
        for name in ("fbx", "fby", "fbz"):
            v = getattr(prob, name)
            if v is not None:
                a = np.ascontiguousarray(prob.field3d(v), dtype=np.float64)
                self._keep.append(a)
                setattr(P, name, _ptr(a))
        P.ov_spinup = int(prob.overland_spinup)
        P.ov_damp_p1, P.ov_damp_p2 = (float(v) for v in prob.spinup_damp)
        self._table = None
        if prob.kr_table:
            method = {"Spline": 0, "Linear": 1}[prob.kr_table[0]]
            self._table = lib().pfo_vgtable_create(method, int(prob.kr_table[1]),
                                                   float(prob.kr_table[2]),
                                                   float(prob.vg_alpha), float(prob.vg_n))
            P.kr_table = self._table
        self.P = P
        self.set_time(prob.start_time + prob.dt if t is None else t)
        s = prob.solver
        S = Settings()
        S.residual_tol, S.step_tol = s.residual_tol, s.step_tol
        S.max_iter, S.krylov_dim, S.max_restarts = s.max_iter, s.krylov_dim, s.max_restarts
        S.eta_choice = ETA[s.eta_choice]
        S.eta_value, S.eta_alpha, S.eta_gamma = s.eta_value, s.eta_alpha, s.eta_gamma
        S.mg_max_levels = s.mg_max_levels
        S.mg_smoother = s.smoother_code()
        S.wjacobi_weight = s.smoother_weight()
        S.use_jacobian = 1 if s.use_jacobian else 0
        S.derivative_epsilon = s.derivative_epsilon
        S.globalization = s.globalization_code()
        S.pc_full = s.pc_matrix_code()
        S.mg_max_iter = s.mg_max_iter
        for q in range(3):
            S.mg_max_min_n[q] = s.mg_max_min_n[q]
        self.S = S

    def __del__(self):
        if getattr(self, "_table", None):
            try:
                lib().pfo_vgtable_destroy(self._table)
            except Exception:
                pass

    def set_time(self, t: float):
        self.t = t
        self._bc = []
        for f, (typ, vals) in enumerate(self.prob.bc_values(t)):
            v = np.ascontiguousarray(vals, dtype=np.float64)
            self._bc.append(v)
            self.P.bc_type[f] = typ
            self.P.bc_val[f] = _ptr(v)

    # ---- functions --------------------------------------------------------
    def residual(self, p, p_old, s_old, dt):
        p, p_old, s_old = (np.ascontiguousarray(x, dtype=np.float64) for x in (p, p_old, s_old))
        f = np.empty_like(p)
        lib().pfo_residual(C.byref(self.P), dt, _ptr(p), _ptr(p_old), _ptr(s_old), _ptr(f))
        return f

    def residual_velocities(self, p, p_old, s_old, dt):
        """F(p) with the face velocities and overland fluxes the evaluation
        writes: (f, vx (nz, ny, nx+1), vy (nz, ny+1, nx), vz (nz+1, ny, nx),
        qx, qy (ny, nx))."""
        p, p_old, s_old = (np.ascontiguousarray(x, dtype=np.float64) for x in (p, p_old, s_old))
        nz, ny, nx = p.shape
        f = np.empty_like(p)
        vx = np.zeros((nz, ny, nx + 1))
        vy = np.zeros((nz, ny + 1, nx))
        vz = np.zeros((nz + 1, ny, nx))
        qx = np.zeros((ny, nx))
        qy = np.zeros((ny, nx))
        out = FluxOut(_ptr(vx), _ptr(vy), _ptr(vz), _ptr(qx), _ptr(qy))
        lib().pfo_residual_out(C.byref(self.P), dt, _ptr(p), _ptr(p_old), _ptr(s_old), _ptr(f),
                               C.byref(out))
        return f, vx, vy, vz, qx, qy

    def saturation(self, p, der=0):
        p = np.ascontiguousarray(p, dtype=np.float64)
        s = np.empty_like(p)
        lib().pfo_saturation(C.byref(self.P), _ptr(p), _ptr(s), der)
        return s

    def relperm(self, p, der=0):
        p = np.ascontiguousarray(p, dtype=np.float64)
        s = np.empty_like(p)
        lib().pfo_relperm(C.byref(self.P), _ptr(p), _ptr(s), der)
        return s

    def jacobian(self, p, dt, symm=0, p_old=None, fd=False):
        """J(p) (7 arrays C W E S N L U) or its PFSymmetric PC form (symm=1:
        C E N U; symm=2: also the (nz, ny) W entries of the i = 0 cells that
        the symmetric storage keeps in a ghost column); p_old is the step's
        old pressure, which only the diffusive overland terms read; fd: the
        matrix the reference builds with Solver.Nonlinear.UseJacobian False
        (no overland surface terms)."""
        p = np.ascontiguousarray(p, dtype=np.float64)
        ns = 4 if symm else 7
        J = [np.empty_like(p) for _ in range(ns)]
        if symm == 2:
            J.append(np.empty(p.shape[:2]))
        arr = (_dp * len(J))(*[_ptr(x) for x in J])
        po = np.ascontiguousarray(p if p_old is None else p_old, dtype=np.float64)
        self.P.ov_p_old = _ptr(po)
        lib().pfo_jacobian_fd(C.byref(self.P), dt, _ptr(p), symm, 1 if fd else 0, arr)
        self.P.ov_p_old = None
        return J

    def matvec(self, J, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        arr = (_dp * 7)(*[_ptr(np.ascontiguousarray(a)) for a in J])
        lib().pfo_matvec7(C.byref(self.P), arr, _ptr(x), _ptr(y))
        return y

    def mg(self):
        return MG(self)

    def newton_solve(self, p_init, p_old, s_old, dt):
        p = np.ascontiguousarray(p_init, dtype=np.float64).copy()
        p_old, s_old = (np.ascontiguousarray(x, dtype=np.float64) for x in (p_old, s_old))
        st = Stats()
        lib().pfo_newton_solve(C.byref(self.P), C.byref(self.S), dt, _ptr(p_old), _ptr(s_old),
                               _ptr(p), C.byref(st))
        return p, st

    def run_time_loop(self, dump_interval: float = 0.0):
        """AdvanceRichards's time loop (solver_richards.c:2075-2090,
        2965-3410, 3700-3720): one SelectTimeStep before the loop, then per
        step SelectTimeStep on the running dt (constant, or growth of it,
        select_time_step.c:58-155, cut to the next cycle transition), the
        dump-time snap and the stop-time cut on every attempt, and on a
        failed solve t and the state put back and dt halved, at most
        Solver.MaxConvergenceFailures attempts.  Returns (pressure per step,
        times, dts, stats per step)."""
        prob = self.prob
        eps = float(np.finfo(np.float32).eps) * 10.0
        g = prob.growth
        stop = prob.stop_time()

        def select(t, dt):
            if g is None:
                dt = float(prob.dt)
            elif dt == 0.0:
                dt = float(g[0])
            else:
                dt = min(max(dt * float(g[1]), float(g[2])), float(g[3]))
            bc_dt = prob.next_transition(t)
            if bc_dt > 0.0 and dt > bc_dt:
                dt = bc_dt
            return dt

        t = float(prob.start_time)
        dump_index = 1.0
        p = prob.initial_pressure().copy()
        dt = select(t, 0.0)
        out_p, times, dts, stats = [], [], [], []
        while t < stop:
            converged, failures = True, 0
            p_old = s_old = None
            while True:
                if converged:
                    dt = select(t, dt)
                    p_old = p.copy()
                    s_old = self.saturation(p_old)
                else:
                    t -= dt
                    half = 0.5 * dt
                    if not (t + half) - t > eps:
                        raise RuntimeError("time increment too small")
                    dt = half
                dump_files = False
                if dump_interval > 0:
                    print_dt = prob.start_time + dump_index * dump_interval - t
                    if dt + eps > print_dt:
                        if abs(dt - print_dt) > eps:
                            dt = print_dt
                        dump_files = True
                if t + dt >= stop:
                    last = stop - t
                    if (t + last) - t > eps:
                        dt = last
                t += dt
                self.set_time(t)
                p_new, st = self.newton_solve(p_old, p_old, s_old, dt)
                converged = st.status in (1, 2)
                if converged:
                    p = p_new
                    break
                failures += 1
                if failures >= prob.solver.max_convergence_failures:
                    raise RuntimeError(f"time step at t = {t} failed {failures} times")
            if dump_files:
                dump_index += 1.0
            out_p.append(p.copy())
            times.append(t)
            dts.append(dt)
            stats.append(st)
        return out_p, times, dts, stats

    def run(self, nsteps=None, callback=None):
        """Advance the problem ``nsteps`` timesteps (AdvanceRichards semantics
        without dt halving).  Returns (pressures per step, stats per step)."""
        prob = self.prob
        plan = prob.time_plan()
        nsteps = len(plan) if nsteps is None else nsteps
        p = prob.initial_pressure().copy()
        out_p, out_s = [], []
        for t, dt in plan[:nsteps]:
            self.set_time(t)
            s_old = self.saturation(p)
            p_new, st = self.newton_solve(p, p, s_old, dt)
            p = p_new
            out_p.append(p.copy())
            out_s.append(st)
            if callback:
                callback(p, st)
        return out_p, out_s


class MG:
    def __init__(self, orc: Oracle):
        self.orc = orc
        self.h = lib().pfo_mg_create(C.byref(orc.P), C.byref(orc.S))

    def __del__(self):
        try:
            lib().pfo_mg_destroy(self.h)
        except Exception:
            pass

    def levels(self):
        out = []
        for l in range(lib().pfo_mg_num_levels(self.h)):
            v = [C.c_int() for _ in range(4)]
            lib().pfo_mg_level_info(self.h, l, *[C.byref(x) for x in v])
            out.append(tuple(x.value for x in v))
        return out

    def setup(self, A4):
        """A4 = C E N U, optionally followed by the i = 0 W plane (jacobian
        with symm=2)."""
        A4 = [np.ascontiguousarray(a, dtype=np.float64) for a in A4]
        self._A = A4
        lib().pfo_mg_set_wghost(self.h, _ptr(A4[4]) if len(A4) > 4 else None)
        arr = (_dp * 4)(*[_ptr(a) for a in A4[:4]])
        lib().pfo_mg_setup(self.h, arr)

    def setup_full(self, A7):
        """A7 = the full Jacobian C W E S N L U (PCMatrixType FullJacobian)."""
        A7 = [np.ascontiguousarray(a, dtype=np.float64) for a in A7]
        self._A = A7
        arr = (_dp * 7)(*[_ptr(a) for a in A7])
        lib().pfo_mg_setup_full(self.h, arr)

    def apply(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        lib().pfo_mg_apply(self.h, _ptr(b), _ptr(x))
        return x
