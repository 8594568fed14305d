"""Richards problem description shared by the CUDA library, the oracle and the
reference CPU build.

A :class:`RichardsProblem` holds what ParFlow's ``ProblemData`` and the
solver keys hold for the path this package accelerates: a box domain with a
structured grid, cell-centred fields (permeability, porosity, specific
storage, van Genuchten parameters, dz multipliers), one boundary condition per
box face, the initial pressure and the KINSOL/GMRES/MGSemi settings.

It produces

* ``to_reference(dir, run)``: the ``.pfidb`` key database plus PFB inputs that
  make ParFlow's own executable solve exactly this problem (key names as read
  by the reference modules, e.g. pfsimulator/parflow_lib/kinsol_nonlin_solver.c:770-968,
  pfsimulator/parflow_lib/problem_saturation.c:884-960, subsrf_sim.c:684-810);
* ``bc_values(t)``: per-face boundary values at time t, computed the way
  ``BCPressure`` does (pfsimulator/parflow_lib/problem_bc_pressure.c:60-615),
  so host code can hand them to the C ABI;
* ``hydrostatic_ic()``: the ``HydroStaticPatch`` initial pressure
  (pfsimulator/parflow_lib/problem_ic_phase_pressure.c:440-672).

Face order everywhere is ParFlow's box patch order: x_lower (Left), x_upper
(Right), y_lower (Down), y_upper (Up), z_lower (Back), z_upper (Front).
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence

import numpy as np

from .pfb import write_pfb
from .pfidb import write_pfidb

FACES = ("x_lower", "x_upper", "y_lower", "y_upper", "z_lower", "z_upper")

# boundary-condition type codes used by the C ABI (include/pfgpu.h)
BC_FLUX = 0          # FluxConst (pfsimulator/parflow_lib/problem_bc_pressure.c:582)
BC_DIRICHLET = 1     # DirEquilRefPatch (problem_bc_pressure.c:143)
BC_OVERLAND_KIN = 2  # OverlandKinematic (bc_pressure_package.c:409)
BC_OVERLAND_DIFF = 3  # OverlandDiffusive (bc_pressure_package.c:427)
BC_OVERLAND = 4       # OverlandFlow (bc_pressure_package.c:354)
BC_SEEPAGE = 5        # SeepageFace (bc_pressure_package.c:392)

_PF_BC_NAME = {BC_FLUX: "FluxConst", BC_DIRICHLET: "DirEquilRefPatch",
               BC_OVERLAND_KIN: "OverlandKinematic",
               BC_OVERLAND_DIFF: "OverlandDiffusive", BC_OVERLAND: "OverlandFlow",
               BC_SEEPAGE: "SeepageFace"}


def pfround(x: float) -> int:
    """ParFlow's rounding macro (pfsimulator/parflow_lib/general.h:176)."""
    return int(x - 0.5) if x < 0.0 else int(x + 0.5)


@dataclass
class BC:
    """Boundary condition on one box face.

    ``values``/``lengths`` describe the face's time cycle: interval i lasts
    ``lengths[i]`` base time units and carries ``values[i]``; ``repeat`` is
    the cycle repeat count (-1 = forever).  For Dirichlet faces the value is
    the pressure on ``ref_patch`` (DirEquilRefPatch).  Flux values are volume
    fluxes per unit area, positive out of the domain on upper faces
    (ParFlow sign convention).
    """

    kind: int
    values: Sequence[float] = (0.0,)
    lengths: Sequence[int] = (1,)
    repeat: int = -1
    ref_patch: str = "z_lower"

    def interval(self, t: float, base_unit: float, start_time: float) -> int:
        """Interval index at time t (time_cycle_data.c:153-199)."""
        cycle_len = int(sum(self.lengths))
        if self.repeat < 0 or t < float(self.repeat * cycle_len * base_unit):
            sub = 1000
            dt_ = pfround(t / (base_unit / sub)) // sub
            ds_ = pfround(start_time / (base_unit / sub)) // sub
            done = int(np.fmod(dt_ - ds_ - 1, cycle_len))
            n = 0
            total = self.lengths[0]
            while done >= total:
                n += 1
                total += self.lengths[n]
            return n
        return len(self.lengths) - 1

    def value_at(self, t, base_unit, start_time) -> float:
        return float(self.values[self.interval(t, base_unit, start_time)])


@dataclass
class SolverSettings:
    """KINSOL / SPGMR / MGSemi settings (keys of kinsol_nonlin_solver.c:770-968,
    kinsol_pc.c:214-246, mg_semi.c:1240-1330)."""

    residual_tol: float = 1e-9
    step_tol: float = 1e-7
    max_iter: int = 15
    krylov_dim: int = 25
    max_restarts: int = 0
    eta_choice: str = "EtaConstant"   # EtaConstant | Walker1 | Walker2
    eta_value: float = 1e-5
    eta_alpha: float = 2.0
    eta_gamma: float = 0.9
    globalization: str = "LineSearch"
    use_jacobian: bool = True
    derivative_epsilon: float = 1e-7  # Solver.Nonlinear.DerivativeEpsilon (J v by differences)
    preconditioner: str = "MGSemi"
    pc_matrix_type: str = "PFSymmetric"
    mg_max_iter: int = 1
    mg_max_levels: int = 100
    # MGSemi.MaxMinNX / NY / NZ: a direction is coarsened only while it has
    # at least max(2 n - 1, 2) cells
    mg_max_min_n: tuple = (1, 1, 1)
    mg_smoother: str = "RedBlackGSPoint"
    # ...MGSemi.Smoother.Symmetric (RedBlackGSPoint: red, black, red when True,
    # red, black when False) and ...MGSemi.Smoother.Weight (WJacobi)
    mg_smoother_symmetric: bool = True
    wjacobi_weight: float = 1.0
    # Solver.Linear.Preconditioner.PFMG.Smoother (pf_pfmg.c:300-305); the
    # other PFMG keys keep their defaults (MaxIter 1, NumPreRelax 1,
    # NumPostRelax 1, RAPType NonGalerkin)
    pfmg_smoother: str = "RBGaussSeidelNonSymmetric"

    def smoother_code(self) -> int:
        """PFGPU_SMOOTH_* of the smoother keys: 0 symmetric red/black
        Gauss-Seidel, 1 weighted Jacobi, 2 non-symmetric red/black.  The
        PFMG preconditioner runs on the same semicoarsening multigrid with
        one pre- and one post-relaxation of its smoother (PFMG's defaults):
        RBGaussSeidelNonSymmetric is one red and one black sweep,
        RBGaussSeidelSymmetric red, black, red, Jacobi a weight-1 Jacobi
        sweep."""
        self.pc_matrix_code()
        if self.preconditioner == "PFMG":
            table = {"RBGaussSeidelNonSymmetric": 2, "RBGaussSeidelSymmetric": 0, "Jacobi": 1}
            if self.pfmg_smoother not in table:
                raise ValueError(f"PFMG smoother {self.pfmg_smoother} is not available")
            return table[self.pfmg_smoother]
        if self.preconditioner != "MGSemi":
            raise ValueError(f"preconditioner {self.preconditioner} is not available")
        if self.mg_smoother == "WJacobi":
            return 1
        if self.mg_smoother != "RedBlackGSPoint":
            raise ValueError(f"unknown MGSemi smoother {self.mg_smoother}")
        return 0 if self.mg_smoother_symmetric else 2

    def pc_matrix_code(self) -> int:
        """Solver.Linear.Preconditioner.PCMatrixType (kinsol_pc.c:215-246):
        1 FullJacobian, 0 the symmetric part.  The type reaches the Jacobian
        evaluation as symm_part, which is only tested for zero
        (richards_jacobian_eval.c:760, 781, 2246): PFSymmetric, SymmetricPart
        and Picard build the same preconditioner matrix."""
        table = {"FullJacobian": 1, "PFSymmetric": 0, "SymmetricPart": 0, "Picard": 0}
        if self.pc_matrix_type not in table:
            raise ValueError(f"PCMatrixType {self.pc_matrix_type} is not available")
        return table[self.pc_matrix_type]

    def globalization_code(self) -> int:
        """Solver.Nonlinear.Globalization (kinsol_nonlin_solver.c:887-905):
        0 LineSearch, 1 InexactNewton."""
        table = {"LineSearch": 0, "InexactNewton": 1}
        if self.globalization not in table:
            raise ValueError(f"Solver.Nonlinear.Globalization {self.globalization} is not available")
        return table[self.globalization]

    def smoother_weight(self) -> float:
        if self.preconditioner == "PFMG":
            return 1.0
        return float(self.wjacobi_weight)
    max_convergence_failures: int = 3


@dataclass
class RichardsProblem:
    nx: int
    ny: int
    nz: int
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 0.5
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    perm: object = 0.01            # float or (nz, ny, nx) array [m/h]
    porosity: float = 0.4
    specific_storage: float = 1e-4
    vg_alpha: object = 2.0         # float or (nz, ny, nx) array [1/m]
    vg_n: object = 3.0
    s_res: float = 0.1
    s_sat: float = 1.0
    gravity: float = 1.0
    density: float = 1.0
    viscosity: float = 1.0
    z_mult: Optional[np.ndarray] = None   # (nz,) dz multipliers, None = 1
    bc: Dict[str, BC] = field(default_factory=dict)
    ic: Optional[np.ndarray] = None       # (nz, ny, nx) initial pressure
    dt: float = 0.1
    nsteps: int = 10
    start_time: float = 0.0
    base_unit: Optional[float] = None     # time-cycle base unit (default dt)
    terrain_following: bool = False
    slope_x: object = 0.0                 # (ny, nx) or float
    slope_y: object = 0.0
    mannings: float = 5.5e-5
    # relative permeability from a lookup table (Geom.domain.RelPerm.
    # NumSamplePoints / MinPressureHead / InterpolationMethod): None or
    # (method "Spline" | "Linear", sample points, min pressure head)
    kr_table: Optional[tuple] = None
    # land-surface sink/source per cell [1/h] (Solver.EvapTransFile /
    # Solver.EvapTrans.FileName): None, a float or an (nz, ny, nx) array
    evap_trans: object = None
    # flow-barrier multipliers of the faces between a cell and its +x / +y /
    # +z neighbour (Solver.Nonlinear.FlowBarrierX/Y/Z, FBx/FBy/FBz.Type
    # PFBFile): None (1 everywhere) or an (nz, ny, nx) array
    fbx: object = None
    fby: object = None
    fbz: object = None
    # OverlandFlowSpinUp (an OverlandFlow top patch drains its ponded head
    # instead of routing it) and OverlandSpinupDampP1 / P2
    overland_spinup: int = 0
    spinup_damp: tuple = (0.0, 0.0)
    # reference output of the face velocities (Solver.PrintVelocities)
    print_velocities: bool = False
    # TimeStep.Type Growth: (initial step, growth factor, min step, max
    # step); None = constant dt.  The time-cycle base unit stays dt.
    growth: Optional[tuple] = None
    solver: SolverSettings = field(default_factory=SolverSettings)
    name: str = "richards"

    # ------------------------------------------------------------------ geometry
    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    def zmult(self) -> np.ndarray:
        if self.z_mult is None:
            return np.ones(self.nz)
        return np.asarray(self.z_mult, dtype=np.float64)

    def rsz(self) -> np.ndarray:
        """Cell-centre elevations, accumulated as problem_real_space_z.c:88-123."""
        zm = self.zmult()
        out = np.empty(self.nz)
        z = float(self.z0)
        for k in range(self.nz):
            z += 0.5 * self.dz * zm[k]
            out[k] = z
            z += 0.5 * self.dz * zm[k]
        return out

    def field3d(self, v) -> np.ndarray:
        if np.isscalar(v):
            return np.full(self.shape, float(v))
        a = np.asarray(v, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        return a

    def field2d(self, v) -> np.ndarray:
        if np.isscalar(v):
            return np.full((self.ny, self.nx), float(v))
        a = np.asarray(v, dtype=np.float64)
        assert a.shape == (self.ny, self.nx)
        return a

    def vg_from_file(self) -> bool:
        return not (np.isscalar(self.vg_alpha) and np.isscalar(self.vg_n))

    # ------------------------------------------------------------------ IC / BC
    def _elevation(self, patch: str) -> float:
        """Elevation of a reference patch (calc_elevations.c for box domains)."""
        if patch == "z_lower":
            return float(self.z0)
        if patch == "z_upper":
            return float(self.z0 + self.dz * float(np.sum(self.zmult())))
        raise ValueError("reference patch must be z_lower or z_upper")

    def hydrostatic_ic(self, value: float, ref_patch: str = "z_lower") -> np.ndarray:
        """HydroStaticPatch IC with constant density: one Newton update of
        F(p) = p - p_ref - rho g (z - z_ref) (problem_ic_phase_pressure.c:440-672)."""
        elev = self._elevation(ref_patch)
        g = -self.gravity
        fcn = (-self.density * g) * (self.rsz() - elev)
        col = value - fcn / 1.0
        return np.broadcast_to(col[:, None, None], self.shape).copy()

    def _dir_equil_values(self, face: str, ref_press: float, ref_patch: str) -> np.ndarray:
        """DirEquilRefPatch values (problem_bc_pressure.c:143-380, constant density)."""
        elev = self._elevation(ref_patch)
        rsz = self.rsz()
        zm = self.zmult()
        dz2 = self.dz * 0.5
        g = -self.gravity
        rho = self.density

        def solve(z):
            pv = ref_press
            fcn = pv - ref_press - 0.5 * (rho + rho) * g * (z - elev)
            if abs(fcn) > 1.0e-6:
                dtmp = 1.0 - 0.5 * 0.0 * g * (z - elev)
                pv = pv - fcn / dtmp
            return pv

        ny, nx, nz = self.ny, self.nx, self.nz
        if face in ("x_lower", "x_upper"):
            out = np.empty((nz, ny))
            for k in range(nz):
                out[k, :] = solve(rsz[k])
        elif face in ("y_lower", "y_upper"):
            out = np.empty((nz, nx))
            for k in range(nz):
                out[k, :] = solve(rsz[k])
        elif face == "z_lower":
            out = np.full((ny, nx), solve(rsz[0] - dz2 * zm[0]))
        else:
            out = np.full((ny, nx), solve(rsz[nz - 1] + dz2 * zm[nz - 1]))
        return out

    def face_shape(self, face: str):
        if face in ("x_lower", "x_upper"):
            return (self.nz, self.ny)
        if face in ("y_lower", "y_upper"):
            return (self.nz, self.nx)
        return (self.ny, self.nx)

    def bc_values(self, t: float):
        """[(type_code, values array of face_shape(face))] for the 6 faces at time t."""
        base = self.base_unit if self.base_unit is not None else self.dt
        out = []
        for face in FACES:
            bc = self.bc.get(face, BC(BC_FLUX, (0.0,)))
            v = bc.value_at(t, base, self.start_time)
            if bc.kind == BC_DIRICHLET:
                out.append((bc.kind, self._dir_equil_values(face, v, bc.ref_patch)))
            else:
                out.append((bc.kind, np.full(self.face_shape(face), v)))
        return out

    def stop_time(self) -> float:
        return float(self.start_time + self.nsteps * self.dt)

    def next_transition(self, t: float) -> float:
        """Time from t to the next interval transition of any face's cycle,
        or -1 (TimeCycleDataComputeNextTransition, time_cycle_data.c:206-297,
        over the BCPressure cycles)."""
        base = self.base_unit if self.base_unit is not None else self.dt
        sub = 1000
        time_eps = float(np.finfo(np.float32).eps) * 10.0
        best = None
        for face in FACES:
            bc = self.bc.get(face, BC(BC_FLUX, (0.0,)))
            lengths = [int(v) for v in bc.lengths]
            if len(lengths) <= 1:
                continue
            clen = sum(lengths)
            stop_defined = bc.repeat * clen * base if bc.repeat > 0 else 1e300
            if not t < stop_defined:
                continue
            dtime = pfround(t / (base / sub)) // sub
            dstart = pfround(self.start_time / (base / sub)) // sub
            n = int((dtime - dstart) / clen)
            done = int(np.fmod(dtime - dstart - 1, clen))
            q, total = 0, lengths[0]
            while done >= total and q + 1 < len(lengths):
                q += 1
                total += lengths[q]
            if (q + 1) % len(lengths) == 0:
                tt = self.start_time + float((n + 1) * clen) * base
            else:
                tt = self.start_time + float(n * clen + total) * base
            if tt < stop_defined:
                best = tt - t if best is None else min(best, tt - t)
        if best is None or not (t + best) - t > time_eps:
            return -1.0
        return best

    def time_plan(self, dump_interval: int = 1):
        """[(t_new, dt)] per timestep, as AdvanceRichards chooses them
        (pfsimulator/parflow_lib/solver_richards.c:3139-3230): constant dt,
        snapped to the next dump time when within TIME_EPSILON
        (general.h:257, FLT_EPSILON * 10) and cut to the stop time on the
        last step; stepping continues while t < stop_time (:4616-4618)."""
        time_eps = float(np.finfo(np.float32).eps) * 10.0
        stop = self.stop_time()
        dump = float(dump_interval * self.dt) if dump_interval > 0 else 0.0
        t = float(self.start_time)
        dump_index = 1.0
        out = []
        while t < stop and len(out) < 10 * self.nsteps + 10:
            dt = float(self.dt)
            if dump > 0:
                print_dt = self.start_time + dump_index * dump - t
                if (dt + time_eps) > print_dt:
                    if abs(dt - print_dt) > time_eps:
                        dt = print_dt
                    dump_index += 1.0
            if (t + dt) >= stop:
                dt = stop - t
            t += dt
            out.append((t, dt))
        return out

    def initial_pressure(self) -> np.ndarray:
        if self.ic is None:
            raise ValueError("problem has no initial pressure")
        return np.asarray(self.ic, dtype=np.float64)

    # ------------------------------------------------------------------ reference
    def to_reference(self, workdir: str, run: Optional[str] = None,
                     dump_interval: int = 1, gpu: Optional[str] = None) -> str:
        """Write ``<run>.pfidb`` and its PFB inputs into ``workdir``.
        dump_interval: > 0 writes pressure and saturation every
        dump_interval * dt of simulated time (TimingInfo.DumpInterval, with
        the dt snapping to dump times that goes with it), < 0 every
        |dump_interval| steps (ParFlow's negative convention,
        solver_richards.c:3165-3170), 0 never.  gpu ("FP64", "Mixed",
        "Mixed16") selects the GPU nonlinear-solver module of a ParFlow build
        that links it (Solver.Nonlinear.GPU)."""
        run = run or self.name
        os.makedirs(workdir, exist_ok=True)
        pj = lambda f: os.path.join(workdir, f)
        k = {}
        k["FileVersion"] = 4
        k["Process.Topology.P"] = 1
        k["Process.Topology.Q"] = 1
        k["Process.Topology.R"] = 1
        k["ComputationalGrid.Lower.X"] = float(self.x0)
        k["ComputationalGrid.Lower.Y"] = float(self.y0)
        k["ComputationalGrid.Lower.Z"] = float(self.z0)
        k["ComputationalGrid.DX"] = float(self.dx)
        k["ComputationalGrid.DY"] = float(self.dy)
        k["ComputationalGrid.DZ"] = float(self.dz)
        k["ComputationalGrid.NX"] = self.nx
        k["ComputationalGrid.NY"] = self.ny
        k["ComputationalGrid.NZ"] = self.nz
        k["GeomInput.Names"] = "domain_input"
        k["GeomInput.domain_input.InputType"] = "Box"
        k["GeomInput.domain_input.GeomName"] = "domain"
        k["Geom.domain.Lower.X"] = float(self.x0)
        k["Geom.domain.Lower.Y"] = float(self.y0)
        k["Geom.domain.Lower.Z"] = float(self.z0)
        k["Geom.domain.Upper.X"] = float(self.x0 + self.nx * self.dx)
        k["Geom.domain.Upper.Y"] = float(self.y0 + self.ny * self.dy)
        k["Geom.domain.Upper.Z"] = float(self.z0 + self.dz * float(np.sum(self.zmult())))
        k["Geom.domain.Patches"] = " ".join(FACES)
        # permeability
        k["Geom.Perm.Names"] = "domain"
        if np.isscalar(self.perm):
            k["Geom.domain.Perm.Type"] = "Constant"
            k["Geom.domain.Perm.Value"] = float(self.perm)
        else:
            write_pfb(pj("perm.pfb"), self.perm, self.dx, self.dy, self.dz, dist=True)
            k["Geom.domain.Perm.Type"] = "PFBFile"
            k["Geom.domain.Perm.FileName"] = "perm.pfb"
        k["Perm.TensorType"] = "TensorByGeom"
        k["Geom.Perm.TensorByGeom.Names"] = "domain"
        for a in "XYZ":
            k[f"Geom.domain.Perm.TensorVal{a}"] = 1.0
        k["SpecificStorage.Type"] = "Constant"
        k["SpecificStorage.GeomNames"] = "domain"
        k["Geom.domain.SpecificStorage.Value"] = float(self.specific_storage)
        k["Phase.Names"] = "water"
        k["Phase.water.Density.Type"] = "Constant"
        k["Phase.water.Density.Value"] = float(self.density)
        k["Phase.water.Viscosity.Type"] = "Constant"
        k["Phase.water.Viscosity.Value"] = float(self.viscosity)
        k["Contaminants.Names"] = ""
        k["Geom.Retardation.GeomNames"] = ""
        k["Gravity"] = float(self.gravity)
        base = self.base_unit if self.base_unit is not None else self.dt
        k["TimingInfo.BaseUnit"] = float(base)
        k["TimingInfo.StartCount"] = 0
        k["TimingInfo.StartTime"] = float(self.start_time)
        k["TimingInfo.StopTime"] = self.stop_time()
        if dump_interval > 0:
            k["TimingInfo.DumpInterval"] = float(dump_interval * self.dt)
        else:
            k["TimingInfo.DumpInterval"] = int(dump_interval) if dump_interval < 0 else -1
        if self.growth is None:
            k["TimeStep.Type"] = "Constant"
            k["TimeStep.Value"] = float(self.dt)
        else:
            # SelectTimeStep growth (select_time_step.c:206-240)
            init, factor, lo, hi = (float(v) for v in self.growth)
            k["TimeStep.Type"] = "Growth"
            k["TimeStep.InitialStep"] = init
            k["TimeStep.GrowthFactor"] = factor
            k["TimeStep.MinStep"] = lo
            k["TimeStep.MaxStep"] = hi
        k["Geom.Porosity.GeomNames"] = "domain"
        k["Geom.domain.Porosity.Type"] = "Constant"
        k["Geom.domain.Porosity.Value"] = float(self.porosity)
        k["Domain.GeomName"] = "domain"
        # van Genuchten
        k["Phase.RelPerm.Type"] = "VanGenuchten"
        k["Phase.RelPerm.GeomNames"] = "domain"
        k["Phase.Saturation.Type"] = "VanGenuchten"
        k["Phase.Saturation.GeomNames"] = "domain"
        if self.vg_from_file():
            write_pfb(pj("vg_alpha.pfb"), self.field3d(self.vg_alpha), self.dx, self.dy, self.dz, dist=True)
            write_pfb(pj("vg_n.pfb"), self.field3d(self.vg_n), self.dx, self.dy, self.dz, dist=True)
            write_pfb(pj("vg_sres.pfb"), self.field3d(self.s_res), self.dx, self.dy, self.dz, dist=True)
            write_pfb(pj("vg_ssat.pfb"), self.field3d(self.s_sat), self.dx, self.dy, self.dz, dist=True)
            k["Phase.RelPerm.VanGenuchten.File"] = 1
            k["Phase.Saturation.VanGenuchten.File"] = 1
            k["Geom.domain.RelPerm.Alpha.Filename"] = "vg_alpha.pfb"
            k["Geom.domain.RelPerm.N.Filename"] = "vg_n.pfb"
            k["Geom.domain.Saturation.Alpha.Filename"] = "vg_alpha.pfb"
            k["Geom.domain.Saturation.N.Filename"] = "vg_n.pfb"
            k["Geom.domain.Saturation.SRes.Filename"] = "vg_sres.pfb"
            k["Geom.domain.Saturation.SSat.Filename"] = "vg_ssat.pfb"
            # region values are still read by the modules' key parsing
            k["Geom.domain.RelPerm.Alpha"] = 1.0
            k["Geom.domain.RelPerm.N"] = 2.0
            k["Geom.domain.Saturation.Alpha"] = 1.0
            k["Geom.domain.Saturation.N"] = 2.0
            k["Geom.domain.Saturation.SRes"] = float(self.s_res)
            k["Geom.domain.Saturation.SSat"] = float(self.s_sat)
        else:
            k["Geom.domain.RelPerm.Alpha"] = float(self.vg_alpha)
            if self.kr_table:
                k["Geom.domain.RelPerm.NumSamplePoints"] = int(self.kr_table[1])
                k["Geom.domain.RelPerm.MinPressureHead"] = float(self.kr_table[2])
                k["Geom.domain.RelPerm.InterpolationMethod"] = str(self.kr_table[0])
            k["Geom.domain.RelPerm.N"] = float(self.vg_n)
            k["Geom.domain.Saturation.Alpha"] = float(self.vg_alpha)
            k["Geom.domain.Saturation.N"] = float(self.vg_n)
            k["Geom.domain.Saturation.SRes"] = float(self.s_res)
            k["Geom.domain.Saturation.SSat"] = float(self.s_sat)
        k["Wells.Names"] = ""
        # time cycles: one per face
        cyc_names = []
        for face in FACES:
            bc = self.bc.get(face, BC(BC_FLUX, (0.0,)))
            cname = f"cyc_{face}"
            cyc_names.append(cname)
            inames = [f"i{i}" for i in range(len(bc.lengths))]
            k[f"Cycle.{cname}.Names"] = " ".join(inames)
            for nm, ln in zip(inames, bc.lengths):
                k[f"Cycle.{cname}.{nm}.Length"] = int(ln)
            k[f"Cycle.{cname}.Repeat"] = int(bc.repeat)
        k["Cycle.Names"] = " ".join(cyc_names)
        k["BCPressure.PatchNames"] = " ".join(FACES)
        for face in FACES:
            bc = self.bc.get(face, BC(BC_FLUX, (0.0,)))
            k[f"Patch.{face}.BCPressure.Type"] = _PF_BC_NAME[bc.kind]
            k[f"Patch.{face}.BCPressure.Cycle"] = f"cyc_{face}"
            if bc.kind == BC_DIRICHLET:
                k[f"Patch.{face}.BCPressure.RefGeom"] = "domain"
                k[f"Patch.{face}.BCPressure.RefPatch"] = bc.ref_patch
            for i, v in enumerate(bc.values):
                k[f"Patch.{face}.BCPressure.i{i}.Value"] = float(v)
        # slopes / mannings
        if np.isscalar(self.slope_x) and np.isscalar(self.slope_y):
            for a, v in (("X", self.slope_x), ("Y", self.slope_y)):
                k[f"TopoSlopes{a}.Type"] = "Constant"
                k[f"TopoSlopes{a}.GeomNames"] = "domain"
                k[f"TopoSlopes{a}.Geom.domain.Value"] = float(v)
        else:
            write_pfb(pj("slope_x.pfb"), self.field2d(self.slope_x), self.dx, self.dy, self.dz, dist=True)
            write_pfb(pj("slope_y.pfb"), self.field2d(self.slope_y), self.dx, self.dy, self.dz, dist=True)
            for a, f in (("X", "slope_x.pfb"), ("Y", "slope_y.pfb")):
                k[f"TopoSlopes{a}.Type"] = "PFBFile"
                k[f"TopoSlopes{a}.GeomNames"] = "domain"
                k[f"TopoSlopes{a}.FileName"] = f
        k["Mannings.Type"] = "Constant"
        k["Mannings.GeomNames"] = "domain"
        k["Mannings.Geom.domain.Value"] = float(self.mannings)
        if self.terrain_following:
            k["Solver.TerrainFollowingGrid"] = True
        # initial condition
        write_pfb(pj("ic_press.pfb"), self.initial_pressure(), self.dx, self.dy, self.dz, dist=True)
        k["ICPressure.Type"] = "PFBFile"
        k["ICPressure.GeomNames"] = "domain"
        k["Geom.domain.ICPressure.FileName"] = "ic_press.pfb"
        k["PhaseSources.water.Type"] = "Constant"
        k["PhaseSources.water.GeomNames"] = "domain"
        k["PhaseSources.water.Geom.domain.Value"] = 0.0
        k["KnownSolution"] = "NoKnownSolution"
        s = self.solver
        k["Solver"] = "Richards"
        k["Solver.MaxIter"] = 100000
        k["Solver.MaxConvergenceFailures"] = s.max_convergence_failures
        k["Solver.Nonlinear.MaxIter"] = s.max_iter
        k["Solver.Nonlinear.ResidualTol"] = s.residual_tol
        k["Solver.Nonlinear.StepTol"] = s.step_tol
        k["Solver.Nonlinear.EtaChoice"] = s.eta_choice
        if s.eta_choice == "EtaConstant":
            k["Solver.Nonlinear.EtaValue"] = s.eta_value
        else:
            k["Solver.Nonlinear.EtaAlpha"] = s.eta_alpha
            k["Solver.Nonlinear.EtaGamma"] = s.eta_gamma
        k["Solver.Nonlinear.UseJacobian"] = bool(s.use_jacobian)
        k["Solver.Nonlinear.DerivativeEpsilon"] = float(s.derivative_epsilon)
        k["Solver.Nonlinear.Globalization"] = s.globalization
        k["Solver.Linear.KrylovDimension"] = s.krylov_dim
        k["Solver.Linear.MaxRestarts"] = s.max_restarts
        k["Solver.Linear.Preconditioner"] = s.preconditioner
        k["Solver.Linear.Preconditioner.PCMatrixType"] = s.pc_matrix_type
        k["Solver.Linear.Preconditioner.MGSemi.MaxIter"] = s.mg_max_iter
        k["Solver.Linear.Preconditioner.MGSemi.MaxLevels"] = s.mg_max_levels
        for axis, n in zip("XYZ", s.mg_max_min_n):
            if n != 1:
                k[f"Solver.Linear.Preconditioner.MGSemi.MaxMinN{axis}"] = n
        if s.preconditioner == "PFMG":
            k["Solver.Linear.Preconditioner.PFMG.Smoother"] = s.pfmg_smoother
        k["Solver.Linear.Preconditioner.MGSemi.Smoother"] = s.mg_smoother
        if s.mg_smoother == "RedBlackGSPoint" and not s.mg_smoother_symmetric:
            k["Solver.Linear.Preconditioner.MGSemi.Smoother.Symmetric"] = "False"
        if s.mg_smoother == "WJacobi" and s.wjacobi_weight != 1.0:
            k["Solver.Linear.Preconditioner.MGSemi.Smoother.Weight"] = float(s.wjacobi_weight)
        if self.evap_trans is not None:
            write_pfb(pj("evap_trans.pfb"), self.field3d(self.evap_trans), self.dx, self.dy,
                      self.dz, dist=True)
            k["Solver.EvapTransFile"] = True
            k["Solver.EvapTrans.FileName"] = "evap_trans.pfb"
        for d, v in (("X", self.fbx), ("Y", self.fby), ("Z", self.fbz)):
            if v is not None:
                fn = f"fb{d.lower()}.pfb"
                write_pfb(pj(fn), self.field3d(v), self.dx, self.dy, self.dz, dist=True)
                k[f"Solver.Nonlinear.FlowBarrier{d}"] = True
                k[f"FB{d.lower()}.Type"] = "PFBFile"
                k[f"Geom.domain.FB{d.lower()}.FileName"] = fn
        if self.overland_spinup:
            k["OverlandFlowSpinUp"] = int(self.overland_spinup)
        if self.spinup_damp != (0.0, 0.0):
            k["OverlandSpinupDampP1"] = float(self.spinup_damp[0])
            k["OverlandSpinupDampP2"] = float(self.spinup_damp[1])
        if self.print_velocities:
            k["Solver.PrintVelocities"] = True
            if any(bc.kind in (BC_OVERLAND_KIN, BC_OVERLAND_DIFF, BC_OVERLAND)
                   for bc in self.bc.values()):
                k["Solver.PrintQxOverland"] = True
                k["Solver.PrintQyOverland"] = True
        k["Solver.PrintSubsurfData"] = False
        k["Solver.PrintPressure"] = dump_interval != 0
        k["Solver.PrintSaturation"] = dump_interval != 0
        k["Solver.PrintMask"] = False
        if gpu:
            k["Solver.Nonlinear.GPU"] = True
            k["Solver.Nonlinear.GPU.Precision"] = gpu
        write_pfidb(k, pj(run + ".pfidb"))
        return run


__all__ = ["RichardsProblem", "BC", "SolverSettings", "FACES",
           "BC_FLUX", "BC_DIRICHLET", "BC_OVERLAND_KIN", "BC_OVERLAND_DIFF", "BC_OVERLAND", "BC_SEEPAGE", "pfround"]
