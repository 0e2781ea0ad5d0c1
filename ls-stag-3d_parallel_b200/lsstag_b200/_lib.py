"""ctypes binding of liblsstag_b200.so (the C ABI in include/lsstag_b200.h).

The library is built in-tree (ls-stag-3d_parallel_b200/lib) by the package
Makefile.  There is no fallback: importing this module without the built
library, or calling it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "liblsstag_b200.so")

LSG_OK = 0
LSG_NOT_CONVERGED = 1
LSG_BREAKDOWN = 2
LSG_ERR_ARG = -1
LSG_ERR_CUDA = -2
LSG_ERR_NOMEM = -3
LSG_ERR_STATE = -4
LSG_ERR_PATTERN = -5
LSG_ERR_SINGULAR = -6

METHOD_FGMRES, METHOD_BICGSTAB = 0, 1
PC_MG, PC_ILU0, PC_NONE = 0, 1, 2
FP64, FP32 = 0, 1
SMOOTHER_ADLJ, SMOOTHER_RBGS = 0, 1
GS_MGS, GS_LOWSYNC = 0, 1
ADLJ_AUTO, ADLJ_REFERENCE, ADLJ_FUSED = 0, 1, 2


class Options(C.Structure):
    _fields_ = [("method", C.c_int), ("precond", C.c_int), ("mg_precision", C.c_int), ("smoother", C.c_int),
                ("n_pre", C.c_int), ("n_post", C.c_int), ("max_levels", C.c_int), ("restart", C.c_int),
                ("max_it", C.c_int), ("zline_reference", C.c_int), ("eps", C.c_double), ("omega", C.c_double),
                ("gram_schmidt", C.c_int), ("adlj_schedule", C.c_int), ("reserved", C.c_int * 6)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("norm_r", C.c_double),
                ("true_residual", C.c_double), ("ms", C.c_double), ("bytes", C.c_double),
                ("vcycles", C.c_int), ("pad", C.c_int), ("kernel_launches", C.c_longlong),
                ("reserved", C.c_int * 4)]


class FlowDesc(C.Structure):
    """lsg_flow_desc (include/lsstag_b200.h)."""
    _fields_ = [("N", C.c_int), ("M", C.c_int), ("K", C.c_int), ("device", C.c_int),
                ("pres", C.c_void_p), ("psolve", C.c_void_p), ("mom", C.c_void_p * 3),
                ("side_type", C.c_void_p), ("vib", C.c_void_p), ("u_w", C.c_void_p), ("theta", C.c_void_p),
                ("delta", C.c_void_p), ("vof", C.c_void_p * 3), ("hflux", C.c_void_p * 3),
                ("bc", C.c_double * 18), ("bc_lap", C.c_double * 5), ("coef", C.c_double), ("coef2", C.c_double),
                ("vbase", C.c_double), ("p_rel_tol", C.c_double), ("zconv_reference", C.c_int),
                ("reserved", C.c_int * 7)]


EXPORTS = [
    "lsg_default_options", "lsg_create", "lsg_destroy", "lsg_last_error", "lsg_set_matrix_csr",
    "lsg_set_matrix_csr_device", "lsg_set_matrix_stencil7", "lsg_setup", "lsg_solve", "lsg_solve_device", "lsg_apply",
    "lsg_precond_apply", "lsg_mg_num_levels", "lsg_mg_level_dims", "lsg_mg_level_csr",
    "lsg_mg_level_tridiag", "lsg_profile_kernel", "lsg_residual_norm_noalloc", "lsg_apply_transpose",
    "lsg_solve_adjoint", "lsg_operator_gradient", "lsg_set_matrix_geometry", "lsg_get_matrix_stencil7",
    "lsg_set_staggered_types", "lsg_projection_rhs", "lsg_projection_rhs_device", "lsg_projection_correct",
    "lsg_projection_correct_device", "lsg_laplace_flux", "lsg_laplace_flux_device", "lsg_projection_adjoint",
    "lsg_momentum_rhs", "lsg_convective_apply", "lsg_convective_apply_device", "lsg_version",
    "lsg_loads_set", "lsg_loads_calculate", "lsg_loads_calculate_device", "lsg_loads_reset_filter",
    "lsg_loads_adjoint", "lsg_loads_adjoint_device", "lsg_set_matrix_helmholtz",
    "lsg_helmholtz_flux", "lsg_convective_flux", "lsg_convective_flux_device", "lsg_momentum_rhs_device",
    "lsg_convective_adjoint", "lsg_convective_adjoint_device", "lsg_gradient_transpose",
    "lsg_gradient_transpose_device", "lsg_projection_adjoint_device", "lsg_tecplot_sol_write",
    "lsg_mesh_build", "lsg_mesh_get", "lsg_mesh_osc_sweeps", "lsg_set_matrix_mesh", "lsg_set_tolerance", "lsg_selftest_wait_limit",
    "lsg_setup_times", "lsg_row_classes",
    "lsg_flow_create", "lsg_flow_destroy", "lsg_flow_last_error", "lsg_flow_set_state", "lsg_flow_step",
    "lsg_flow_state",
    "lsg_momentum_cotangents_device", "lsg_fluid_faces_device", "lsg_clamp_transpose_device",
    "lsg_scatter_add_device", "lsg_axpy_device",
    "lsg_tecplot_sol_async", "lsg_tecplot_wait",
]

_lib = None


class LoadsResult(C.Structure):
    """lsg_loads_result: sums of the cut-cell forces, coefficients, raw and
    filtered moments (M_z, M_x, M_y)."""
    _fields_ = [("force", C.c_double * 3), ("coef", C.c_double * 3), ("moment_raw", C.c_double * 3),
                ("moment", C.c_double * 3), ("count", C.c_int)]


class LsgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lsstag_b200 error {code}: {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built (run make in {PKG_ROOT})")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    ip = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    lib.lsg_default_options.argtypes = [C.POINTER(Options)]
    lib.lsg_default_options.restype = None
    lib.lsg_create.argtypes = [C.c_int, C.POINTER(P)]
    lib.lsg_destroy.argtypes = [P]
    lib.lsg_last_error.argtypes = [P]
    lib.lsg_last_error.restype = C.c_char_p
    lib.lsg_set_matrix_csr.argtypes = [P, C.c_int, C.c_int, C.c_int, ip, ip, dp]
    lib.lsg_set_matrix_csr_device.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P, P, C.c_longlong]
    lib.lsg_set_matrix_stencil7.argtypes = [P, C.c_int, C.c_int, C.c_int, dp]
    lib.lsg_setup.argtypes = [P, C.POINTER(Options)]
    lib.lsg_solve.argtypes = [P, dp, dp, C.POINTER(Stats)]
    lib.lsg_solve_device.argtypes = [P, P, P, C.POINTER(Stats)]
    lib.lsg_apply.argtypes = [P, dp, dp]
    lib.lsg_precond_apply.argtypes = [P, dp, dp]
    lib.lsg_mg_num_levels.argtypes = [P]
    lib.lsg_mg_level_dims.argtypes = [P, C.c_int, ip]
    lib.lsg_mg_level_csr.argtypes = [P, C.c_int, ip, ip, dp, C.POINTER(C.c_longlong)]
    lib.lsg_mg_level_tridiag.argtypes = [P, C.c_int, C.c_char, dp, dp, dp]
    lib.lsg_profile_kernel.argtypes = [P, C.c_int, C.c_int, dp, dp]
    lib.lsg_residual_norm_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, P, P, P, P, P, P]
    lib.lsg_apply_transpose.argtypes = [P, dp, dp]
    lib.lsg_solve_adjoint.argtypes = [P, dp, dp, C.POINTER(Stats)]
    lib.lsg_operator_gradient.argtypes = [P, dp, dp, dp]
    lib.lsg_set_matrix_geometry.argtypes = [P, C.c_int, C.c_int, C.c_int, ip, dp, dp, dp, dp, dp, C.c_longlong,
                                            C.c_longlong]
    lib.lsg_get_matrix_stencil7.argtypes = [P, dp]
    lib.lsg_set_staggered_types.argtypes = [P, ip, ip, ip]
    lib.lsg_laplace_flux.argtypes = [P, ip, dp, dp, dp, dp, dp]
    lib.lsg_convective_apply.argtypes = [P, C.c_int, dp, dp, dp, dp, dp, dp, C.c_int]
    lib.lsg_convective_apply_device.argtypes = [P, C.c_int] + [C.c_void_p] * 6 + [C.c_int]
    lib.lsg_momentum_rhs.argtypes = [P, C.c_int, ip, ip, dp, dp, dp, dp, dp, dp, dp, dp, C.c_double, dp, dp]
    lib.lsg_projection_adjoint.argtypes = [P, dp, dp, dp, dp, C.c_double, dp, dp, dp, dp, C.POINTER(Stats)]
    lib.lsg_gradient_transpose.argtypes = [P, dp, dp, dp, dp]
    lib.lsg_gradient_transpose_device.argtypes = [P] + [C.c_void_p] * 4
    lib.lsg_tecplot_sol_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, dp, dp, dp, ip, dp, dp, dp, dp,
                                          dp, dp, C.c_int]
    lib.lsg_tecplot_sol_async.argtypes = [P, C.c_char_p, dp, dp, dp, ip] + [C.c_void_p] * 4 + [dp, dp, C.c_int]
    lib.lsg_tecplot_wait.argtypes = [P]
    lib.lsg_projection_adjoint_device.argtypes = ([P] + [C.c_void_p] * 4 + [C.c_double] + [C.c_void_p] * 4
                                                  + [C.POINTER(Stats)])
    lib.lsg_laplace_flux_device.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, dp, C.c_void_p, C.c_void_p]
    lib.lsg_projection_rhs.argtypes = [P, dp, dp, dp, dp, dp]
    lib.lsg_projection_rhs_device.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lsg_projection_correct.argtypes = [P, dp, dp, dp, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_int]
    lib.lsg_projection_correct_device.argtypes = [P] + [C.c_void_p] * 8 + [C.c_double, C.c_double, C.c_int]
    lib.lsg_set_matrix_helmholtz.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, ip] + [dp] * 11 + [
        C.c_double, C.c_double, C.c_int]
    lib.lsg_helmholtz_flux.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, ip, dp, dp, dp, C.c_double, C.c_int,
                                       ip] + [dp] * 12 + [dp]
    lib.lsg_convective_flux.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int] + [dp] * 7 + [dp]
    lib.lsg_convective_flux_device.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 6 + [
        dp, C.c_void_p]
    lib.lsg_momentum_rhs_device.argtypes = [P, C.c_int] + [C.c_void_p] * 7 + [C.c_double] + [C.c_void_p] * 3
    lib.lsg_convective_adjoint.argtypes = [P, C.c_int] + [dp] * 9 + [C.c_int]
    lib.lsg_convective_adjoint_device.argtypes = [P, C.c_int] + [C.c_void_p] * 9 + [C.c_int]
    lib.lsg_loads_set.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip] + [dp] * 8 + [C.c_double,
                                                                                             C.c_double]
    lib.lsg_loads_calculate.argtypes = [P] + [dp] * 8 + [C.c_double, dp, C.POINTER(LoadsResult)]
    lib.lsg_loads_calculate_device.argtypes = [P] + [C.c_void_p] * 8 + [C.c_double, C.c_void_p,
                                                                        C.POINTER(LoadsResult)]
    lib.lsg_loads_reset_filter.argtypes = [P, C.c_double]
    lib.lsg_loads_adjoint.argtypes = [P, dp, dp, C.c_double, dp, dp, dp, dp]
    lib.lsg_loads_adjoint_device.argtypes = [P, dp, C.c_void_p, C.c_double] + [C.c_void_p] * 4
    lib.lsg_mesh_build.argtypes = [P, C.c_int, C.c_int, C.c_int, dp, ip, C.c_int, dp, dp, dp]
    lib.lsg_mesh_get.argtypes = [P, C.c_int, C.c_void_p]
    lib.lsg_mesh_osc_sweeps.argtypes = [P]
    lib.lsg_set_matrix_mesh.argtypes = [P, C.c_longlong, C.c_longlong]
    lib.lsg_set_tolerance.argtypes = [P, C.c_double]
    lib.lsg_selftest_wait_limit.argtypes = [P]
    lib.lsg_setup_times.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.lsg_row_classes.argtypes = [P, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.lsg_flow_create.argtypes = [C.POINTER(FlowDesc), C.POINTER(C.c_void_p)]
    lib.lsg_flow_destroy.argtypes = [P]
    lib.lsg_flow_last_error.argtypes = [P]
    lib.lsg_flow_last_error.restype = C.c_char_p
    lib.lsg_flow_set_state.argtypes = [P, C.c_void_p * 3, C.c_void_p * 3, C.c_void_p, C.c_void_p]
    lib.lsg_flow_step.argtypes = [P, C.POINTER(C.c_int)]
    lib.lsg_flow_state.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lsg_momentum_cotangents_device.argtypes = [P, C.c_int, P, P, C.c_double] + [P] * 6
    lib.lsg_fluid_faces_device.argtypes = [P, C.c_int, P, P]
    lib.lsg_clamp_transpose_device.argtypes = [P] + [C.c_void_p] * 8
    lib.lsg_scatter_add_device.argtypes = [P, C.c_longlong] + [C.c_void_p] * 7
    lib.lsg_axpy_device.argtypes = [P, C.c_longlong, C.c_double, C.c_void_p, C.c_void_p]
    lib.lsg_version.restype = C.c_char_p
    _lib = lib
    return lib


def default_options(**over) -> Options:
    o = Options()
    load().lsg_default_options(C.byref(o))
    for k, v in over.items():
        setattr(o, k, v)
    return o


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Context:
    """Owns one lsg_ctx (one device, one operator)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.h = C.c_void_p()
        rc = self.lib.lsg_create(device, C.byref(self.h))
        if rc != LSG_OK:
            raise LsgError(rc, "lsg_create failed (no usable CUDA device?)")

    def check(self, rc):
        if rc < 0:
            raise LsgError(rc, self.lib.lsg_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self.lib.lsg_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
