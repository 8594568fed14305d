"""ctypes binding of libpfgpu.so (the C ABI declared in include/pfgpu.h).

The library is the product path: there is no CPU fallback.  Loading fails
loudly when the shared object is missing or was built for another ABI.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfgpu.so")

ABI_VERSION = 2
PREC_FP64, PREC_MIXED, PREC_MIXED_H16 = 0, 1, 2
BC_FLUX, BC_DIRICHLET, BC_OVERLAND_KIN, BC_OVERLAND_DIFF, BC_OVERLAND, BC_SEEPAGE = \
    0, 1, 2, 3, 4, 5
FIELD_PERM_X, FIELD_PERM_Y, FIELD_PERM_Z = 0, 1, 2
FIELD_VG_ALPHA, FIELD_VG_N, FIELD_S_RES, FIELD_S_SAT = 3, 4, 5, 6
FIELD_FB_X, FIELD_FB_Y, FIELD_FB_Z = 7, 8, 9
OK, NOT_CONVERGED = 0, 1

_dp = C.POINTER(C.c_double)


class Desc(C.Structure):
    _fields_ = [("abi_version", C.c_int),
                ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("gravity", C.c_double), ("viscosity", C.c_double), ("density", C.c_double),
                ("porosity", C.c_double), ("specific_storage", C.c_double),
                ("vg_alpha", C.c_double), ("vg_n", C.c_double),
                ("s_res", C.c_double), ("s_sat", C.c_double),
                ("vg_from_file", C.c_int),
                ("z_mult", _dp),
                ("precision", C.c_int),
                ("residual_tol", C.c_double), ("step_tol", C.c_double),
                ("max_iter", C.c_int), ("krylov_dim", C.c_int), ("max_restarts", C.c_int),
                ("eta_choice", C.c_int),
                ("eta_value", C.c_double), ("eta_alpha", C.c_double), ("eta_gamma", C.c_double),
                ("mg_max_levels", C.c_int), ("mg_smoother", C.c_int),
                ("wjacobi_weight", C.c_double),
                ("mg_max_min_n", C.c_int * 3)]


class Stats(C.Structure):
    _fields_ = [("kinsol_status", C.c_int),
                ("nonlin_iters", C.c_int), ("lin_iters", C.c_int), ("fevals", C.c_int),
                ("pc_setups", C.c_int), ("pc_solves", C.c_int),
                ("lin_conv_fails", C.c_int), ("beta_cond_fails", C.c_int),
                ("backtracks", C.c_int), ("fnorm", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# every symbol include/pfgpu.h declares
EXPORTS = ["pfgpu_create", "pfgpu_destroy", "pfgpu_last_error", "pfgpu_set_field",
           "pfgpu_set_bc", "pfgpu_nl_function_eval", "pfgpu_jacobian_matvec",
           "pfgpu_pc_setup", "pfgpu_pc_apply", "pfgpu_saturation", "pfgpu_newton_solve",
           "pfgpu_set_pressure", "pfgpu_get_pressure", "pfgpu_advance", "pfgpu_mg_levels",
           "pfgpu_stream", "pfgpu_kernel_launches", "pfgpu_time_kernel",
           "pfgpu_residual_noalloc", "pfgpu_ensemble_advance", "pfgpu_set_surface",
           "pfgpu_adjoint_record", "pfgpu_adjoint_gradient", "pfgpu_write_pfb",
           "pfgpu_read_pfb", "pfgpu_set_bc_cycle", "pfgpu_set_time_step", "pfgpu_run",
           "pfgpu_newton_solve_sat", "pfgpu_set_old_pressure", "pfgpu_autotune",
           "pfgpu_set_jacobian_mode", "pfgpu_set_relperm_table", "pfgpu_set_evap_trans",
           "pfgpu_face_velocities", "pfgpu_solve_graph", "pfgpu_set_globalization",
           "pfgpu_set_pc_matrix", "pfgpu_set_mg_max_iter",
           "pfgpu_set_overland_spinup"]
PFB_PRESSURE, PFB_SATURATION = 100, 101
KERNELS = {"residual": 0, "jacobian": 1, "matvec": 2, "rb_smooth": 3, "vcycle": 4, "mg_setup": 5,
           "colour_sweep": 6}

_lib = None


def load(path: str = LIB_PATH):
    """Load libpfgpu.so and declare its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m parflow_b200.build`")
    L = C.CDLL(path)
    vp = C.c_void_p
    L.pfgpu_create.argtypes = [C.POINTER(Desc), C.c_int]
    L.pfgpu_create.restype = vp
    L.pfgpu_destroy.argtypes = [vp]
    L.pfgpu_destroy.restype = None
    L.pfgpu_last_error.restype = C.c_char_p
    L.pfgpu_set_field.argtypes = [vp, C.c_int, C.c_void_p]
    L.pfgpu_set_bc.argtypes = [vp, C.c_int, C.c_int, C.c_void_p]
    L.pfgpu_adjoint_record.argtypes = [vp, C.c_int]
    L.pfgpu_adjoint_gradient.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.c_int,
                                         C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                         C.c_double, C.POINTER(C.c_double), vp, vp, vp]
    L.pfgpu_set_surface.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double]
    L.pfgpu_write_pfb.argtypes = [vp, C.c_int, C.c_char_p, C.c_double, C.c_double, C.c_double]
    L.pfgpu_set_bc_cycle.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int,
                                     C.c_double, C.c_double]
    L.pfgpu_set_time_step.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int]
    L.pfgpu_run.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_int,
                            C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(Stats),
                            C.POINTER(C.c_int)]
    L.pfgpu_read_pfb.argtypes = [vp, C.c_int, C.c_char_p]
    L.pfgpu_nl_function_eval.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                         C.c_void_p]
    L.pfgpu_jacobian_matvec.argtypes = [vp, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    L.pfgpu_pc_setup.argtypes = [vp, C.c_void_p, C.c_double]
    L.pfgpu_set_old_pressure.argtypes = [vp, C.c_void_p]
    L.pfgpu_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
    L.pfgpu_set_jacobian_mode.argtypes = [vp, C.c_int, C.c_double]
    L.pfgpu_set_relperm_table.argtypes = [vp, C.c_int, C.c_int, C.c_double]
    L.pfgpu_pc_apply.argtypes = [vp, C.c_void_p, C.c_void_p]
    L.pfgpu_set_evap_trans.argtypes = [vp, C.c_void_p]
    L.pfgpu_solve_graph.argtypes = [vp, C.c_int]
    L.pfgpu_set_globalization.argtypes = [vp, C.c_int]
    L.pfgpu_set_pc_matrix.argtypes = [vp, C.c_int]
    L.pfgpu_set_mg_max_iter.argtypes = [vp, C.c_int]
    L.pfgpu_set_overland_spinup.argtypes = [vp, C.c_int, C.c_double, C.c_double]
    L.pfgpu_face_velocities.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double] + \
        [C.c_void_p] * 5
    L.pfgpu_saturation.argtypes = [vp, C.c_void_p, C.c_void_p]
    L.pfgpu_newton_solve.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                     C.POINTER(Stats)]
    L.pfgpu_newton_solve_sat.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                         C.c_void_p, C.POINTER(Stats)]
    L.pfgpu_set_pressure.argtypes = [vp, C.c_void_p]
    L.pfgpu_get_pressure.argtypes = [vp, C.c_void_p]
    L.pfgpu_advance.argtypes = [vp, C.c_double, C.c_int, C.POINTER(Stats)]
    L.pfgpu_mg_levels.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
    L.pfgpu_stream.argtypes = [vp]
    L.pfgpu_stream.restype = vp
    L.pfgpu_kernel_launches.argtypes = [vp]
    L.pfgpu_kernel_launches.restype = C.c_longlong
    L.pfgpu_time_kernel.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
    L.pfgpu_ensemble_advance.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(C.c_double), C.c_int,
                                         C.c_int, C.POINTER(Stats), C.POINTER(C.c_int)]
    L.pfgpu_residual_noalloc.argtypes = [C.POINTER(Desc)] + [vp] * 5 + \
        [C.POINTER(C.c_int), C.POINTER(C.c_void_p)] + [vp] * 3 + [C.c_double, vp, vp]
    _lib = L
    return L


def last_error() -> str:
    return load().pfgpu_last_error().decode(errors="replace")


class PfgpuError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc < 0:
        raise PfgpuError(f"{what} failed ({rc}): {last_error()}")
    return rc
