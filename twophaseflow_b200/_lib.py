"""ctypes binding of the in-tree CUDA library ``libtpf.so`` (C ABI in include/tpf.h).

The library is the only compute path: if it is missing or no CUDA device is
visible, every entry point raises.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtpf.so")

TPF_OK, TPF_EINVAL, TPF_ENOCONV, TPF_ECUDA, TPF_EABORT, TPF_ESINGULAR = range(6)
TPF_F64, TPF_F32 = 0, 1
TPF_BC_WALL, TPF_BC_PERIODIC = 0, 1
TPF_CCD_APPLY_METRIC = 1
TPF_PPE_CG, TPF_PPE_GMRES = 0, 1
TPF_PRECOND_NONE, TPF_PRECOND_JACOBI, TPF_PRECOND_LINE, TPF_PRECOND_LINE_PCR = range(4)
TPF_PREC_F64, TPF_PREC_MIXED = 0, 1
TPF_PPE_STATIC_MAX_DOF, TPF_PPE_STATIC_MAX_AXIS = 66049, 4097


class tpf_ppe_options(C.Structure):
    _fields_ = [
        ("method", C.c_int),
        ("precond", C.c_int),
        ("precision", C.c_int),
        ("tol", C.c_double),
        ("maxiter", C.c_int64),
        ("restart", C.c_int),
        ("c_tau", C.c_double),
        ("pcr_stages", C.c_int),
        ("inner_tol", C.c_double),
        ("max_refine", C.c_int64),
    ]


class tpf_ppe_result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("applies", C.c_int64),
        ("refinements", C.c_int64),
        ("rel_residual", C.c_double),
        ("info", C.c_int),
    ]


class tpf_fccd_ppe_options(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("maxiter", C.c_int64),
        ("restart", C.c_int),
        ("precond", C.c_int),
    ]


class tpf_learned_options(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("maxiter", C.c_int64),
        ("smooth", C.c_int),
        ("omega", C.c_double),
        ("check_every", C.c_int),
        ("stall_checks", C.c_int),
        ("stall_factor", C.c_double),
        ("fallback", C.c_int),
        ("use_graph", C.c_int),
        ("window", C.c_int),
        ("outer", C.c_int),
        ("restart", C.c_int),
    ]


class tpf_lppe_result(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("fallback_iterations", C.c_int64),
        ("restarts", C.c_int64),
        ("rel_residual", C.c_double),
        ("info", C.c_int),
        ("fell_back", C.c_int),
    ]


# name -> (restype, argtypes); every function declared in include/tpf.h
SIGNATURES = {
    "tpf_version": (C.c_int, []),
    "tpf_last_error": (C.c_char_p, []),
    "tpf_set_launch_autotune": (C.c_int, [C.c_int]),
    "tpf_launch_autotune_entries": (C.c_int, []),
    "tpf_ccd_plan_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int64, C.c_double, C.c_int, C.c_int]),
    "tpf_ccd_plan_destroy": (C.c_int, [C.c_void_p]),
    "tpf_ccd_plan_set_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "tpf_ccd_plan_set_metric": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "tpf_ccd_apply": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_void_p]),
    "tpf_ccd_apply_refined": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "tpf_ccd_apply_vd": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "tpf_ccd_apply_corrector": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_cfl_maxima": (C.c_int, [C.c_int64, C.c_int, C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_int,
                                 C.c_void_p, C.c_void_p]),
    "tpf_dccd_filter": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.c_double, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_curvature_psi": (C.c_int, [C.c_int, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p), C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_gaussian3x3": (C.c_int, [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_update_properties": (C.c_int, [C.c_int64, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_rc_divergence_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_fccd_ppe_default_options": (None, [C.c_void_p]),
    "tpf_fccd_ppe_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int64),
                                      C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                      C.c_int64, C.c_void_p]),
    "tpf_fccd_ppe_destroy": (C.c_int, [C.c_void_p]),
    "tpf_fccd_ppe_set_options": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tpf_fccd_ppe_prepare": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_fccd_ppe_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_fccd_ppe_diag_inv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_fccd_ppe_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "tpf_fccd_product": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_fccd_node_gradient_axis_nonuniform": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_void_p,
                                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                           C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_fccd_flux_divergence_axis_nonuniform": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int,
                                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                             C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_fccd_node_gradient_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_double, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_fccd_flux_divergence_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_double,
                                                C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_tvd_rk3_stage": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                    C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_sync_periodic_images": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.c_void_p, C.c_int,
                                           C.c_void_p]),
    "tpf_reinit_compression_flux": (C.c_int, [C.c_int, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_void_p), C.c_int, C.c_void_p]),
    "tpf_reinit_filtered_divergence_axis_metric": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int,
                                                               C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                                                               C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_reinit_filtered_divergence_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_double,
                                                      C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_reinit_cn_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_double, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_mass_sums": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_mass_correction_apply": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_void_p]),
    "tpf_visc_lowfd_axis": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                      C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_visc_stress": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_visc_band_masks": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p,
                                      C.POINTER(C.c_void_p), C.c_int, C.c_void_p]),
    "tpf_visc_select": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                  C.c_void_p]),
    "tpf_visc_band_finalize": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_visc_accumulate": (C.c_int, [C.c_int64, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_void_p,
                                      C.c_int, C.c_void_p]),
    "tpf_cn_predictor_combine": (C.c_int, [C.c_int64, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_uccd6_accumulate": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_ns_conv_accumulate": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                         C.c_void_p]),
    "tpf_ns_scaled": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int,
                                C.c_void_p]),
    "tpf_ns_explicit_rhs": (C.c_int, [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tpf_ccd_enforce_wall_neumann": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
    "tpf_ppe_default_options": (None, [C.POINTER(tpf_ppe_options)]),
    "tpf_ppe_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int64),
                                 C.POINTER(C.POINTER(C.c_double)), C.c_int64, C.POINTER(tpf_ppe_options)]),
    "tpf_ppe_destroy": (C.c_int, [C.c_void_p]),
    "tpf_ppe_set_options": (C.c_int, [C.c_void_p, C.POINTER(tpf_ppe_options)]),
    "tpf_ppe_read_result": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_ppe_set_cg_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "tpf_ppe_prepare": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_ppe_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_ppe_precondition": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_ppe_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(tpf_ppe_result)]),
    "tpf_ppe_solve_batched": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p,
                                        C.POINTER(tpf_ppe_result)]),
    "tpf_ppe_solve_cg_static": (C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_double)),
                                          C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_double, C.c_int64, C.c_void_p, C.POINTER(tpf_ppe_result)]),
    "tpf_unet_num_params": (C.c_int64, []),
    "tpf_unet_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int]),
    "tpf_unet_destroy": (C.c_int, [C.c_void_p]),
    "tpf_unet_set_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "tpf_unet_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "tpf_unet_set_forward_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "tpf_unet_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_unet_backward": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_unet_train_step": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                      C.POINTER(C.c_double), C.c_void_p]),
    "tpf_unet_train_step_energy": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                             C.c_int, C.c_float, C.c_float, C.POINTER(C.c_double), C.c_void_p]),
    "tpf_lppe_default_options": (None, [C.POINTER(tpf_learned_options)]),
    "tpf_lppe_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_int]),
    "tpf_lppe_destroy": (C.c_int, [C.c_void_p]),
    "tpf_lppe_prepare": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpf_lppe_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(tpf_learned_options), C.c_void_p, C.POINTER(tpf_lppe_result)]),
    "tpf_lppe_precondition": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "tpf_lppe_set_smooth_block": (C.c_int, [C.c_void_p, C.c_int]),
    "tpf_lppe_smooth": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "tpf_lppe_pair": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    "tpf_lppe_pair_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_void_p]),
}

_lib = None
_lock = threading.Lock()


class LibraryNotBuilt(RuntimeError):
    pass


def load(path: str | None = None):
    """Load libtpf.so (once) and attach prototypes.  Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise LibraryNotBuilt(
                f"{p} is missing: build it with `python -m twophaseflow_b200.build` "
                "(the CUDA library is the only compute path; there is no CPU fallback)")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().tpf_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = ""):
    """Map a tpf status code to the reference's exception types."""
    if status == TPF_OK:
        return
    msg = last_error() or what
    if status == TPF_EINVAL:
        raise ValueError(msg)
    if status == TPF_ESINGULAR:
        raise np.linalg.LinAlgError(msg)
    raise RuntimeError(msg)


def dptr(t) -> C.c_void_p:
    return C.c_void_p(int(t.data_ptr()))


def current_stream_handle():
    import torch
    return C.c_void_p(int(torch.cuda.current_stream().cuda_stream))
