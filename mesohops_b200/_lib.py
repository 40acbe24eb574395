"""ctypes binding of ``libhops_b200.so`` (C ABI in ``include/hops_b200.h``).

The library is built in-tree (``mesohops_b200/lib``) by ``mesohops_b200.build``.
There is no fallback: if the shared library is missing or fails to load, every
GPU entry point raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os

from .exceptions import TrajectoryError, UnsupportedRequest

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libhops_b200.so")

HOPS_OK, HOPS_EINVAL, HOPS_ECUDA, HOPS_ENOTSUP, HOPS_ENONFINITE = 0, 1, 2, 3, 5
HOPS_ETIMEOUT = 6
PREC_C128, PREC_C64, PREC_MIXED = 0, 1, 2
EOM_CODES = {"NORMALIZED NONLINEAR": 0, "NONLINEAR": 1, "LINEAR": 2}

_p = C.c_void_p
_i = C.c_int32


class HopsStructure(C.Structure):
    """Mirror of ``hops_structure`` (all pointer fields are device pointers)."""
    _fields_ = [
        ("n_hier", _i), ("n_state", _i), ("n_mode", _i), ("n_lop", _i),
        ("n_first", _i), ("n_up", _i), ("n_dn", _i), ("site_projector", _i),
        ("max_up", _i), ("max_dn", _i),
        ("k_decay", _p), ("k_decay_f", _p),
        ("up_ptr", _p), ("up_aux", _p), ("up_mode", _p),
        ("dn_ptr", _p), ("dn_aux", _p), ("dn_mode", _p), ("dn_coef", _p), ("dn_coef_f", _p),
        ("mode_lop", _p), ("mode_g", _p), ("mode_w", _p), ("mode_gw", _p), ("mode_gw_f", _p),
        ("first_aux", _p), ("first_mode", _p),
        ("l_ptr", _p), ("l_col", _p), ("l_val", _p), ("l_val_f", _p),
        ("lh_ptr", _p), ("lh_col", _p), ("lh_val", _p), ("lh_val_f", _p),
        ("lop_active", _p), ("lop_site", _p), ("lop_sval", _p),
        ("h_ptr", _p), ("h_col", _p), ("h_val", _p), ("h_val_f", _p),
        ("mode_site", _p), ("mode_gwv", _p), ("mode_gwv_f", _p),
        ("dn_coef_site", _p), ("dn_coef_site_f", _p),
        ("up_site", _p), ("dn_site", _p), ("h_diag", _p),
        ("lt_coef", _p), ("l2_ptr", _p), ("l2_col", _p), ("l2_val", _p),
        ("n_up_prefix", _i), ("reserved", _i),
    ]


class HopsBatch(C.Structure):
    """Mirror of ``hops_batch``."""
    _fields_ = [
        ("n_traj", _i), ("precision", _i), ("eom", _i), ("n_t1", _i), ("n_t2", _i),
        ("phi", _p), ("acc", _p), ("y0", _p), ("y1", _p),
        ("zmem", _p), ("work", _p), ("noise1", _p), ("noise2", _p), ("status", _p),
        ("phi_lo", _p), ("defer_scale", _i), ("noise_c128", _i),
    ]


class HopsTask(C.Structure):
    """Mirror of ``hops_task``."""
    _fields_ = [
        ("st", _p), ("phi", _p), ("zmem", _p), ("noise1", _p), ("noise2", _p),
        ("psi_out", _p), ("scratch", _p),
        ("n_t1", _i), ("n_t2", _i), ("it0", _i), ("di", _i), ("n_steps", _i),
        ("precision", _i), ("eom", _i), ("status", _i),
        ("tau_over_hbar", C.c_double), ("scale", C.c_double),
        ("noise_c128", _i), ("pad", _i),
    ]


class HopsFluxTask(C.Structure):
    """Mirror of ``hops_flux_task``."""
    _fields_ = [
        ("st", _p), ("phi", _p), ("zmem", _p), ("z1", _p), ("z2", _p), ("aux_mask", _p),
        ("e_deriv", _p), ("e_up", _p), ("e_down", _p), ("k_aux", _p), ("dt", C.c_double),
        ("eom", _i), ("pad", _i),
    ]


class HopsStructureDesc(C.Structure):
    """Mirror of ``hops_structure_desc`` (all pointer fields are host pointers)."""
    _fields_ = [
        ("n_hier", _i), ("n_state", _i), ("n_mode", _i), ("n_lop", _i),
        ("up_ptr", _p), ("up_aux", _p), ("up_mode", _p),
        ("dn_ptr", _p), ("dn_aux", _p), ("dn_mode", _p), ("dn_k", _p),
        ("mode_lop", _p), ("mode_g", _p), ("mode_w", _p), ("lops", _p),
        ("hamiltonian", _p), ("lt_coef", _p),
    ]


_lib = None


def lib():
    """Load (once) and return the CUDA library; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"mesohops_b200 CUDA library not found at {LIB_PATH}; "
            "build it with `python -m mesohops_b200.build` (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.hops_last_error.restype = C.c_char_p
    L.hops_version.restype = C.c_int
    L.hops_device_query.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.hops_scalar_workspace_doubles.restype = C.c_size_t
    L.hops_scalar_workspace_doubles.argtypes = [_i, _i, _i, _i]
    L.hops_batch_reset.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _p]
    L.hops_dsystem_dt.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _p, _p, _p,
                                  _p, _p]
    L.hops_rk4_propagate.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _i, _i,
                                     _i, C.c_double, _p, _p]
    L.hops_resident_propagate.argtypes = [_p, _i, _i, _i, _i, _i, _p]
    L.hops_resident_scalar_doubles.restype = _i
    L.hops_resident_scalar_doubles.argtypes = [_i, _i, _i]
    L.hops_noise_filter.argtypes = [_p, _p, _i, _i, _p, _p, _p, C.POINTER(C.c_int64), _p]
    L.hops_noise_filter_shared.argtypes = [_p, _i, _p, _i, _i, _p, _p, _p,
                                           C.POINTER(C.c_int64), _p]
    L.hops_noise_filter_work_doubles.restype = C.c_size_t
    L.hops_noise_filter_work_doubles.argtypes = [_i, _i]
    L.hops_noise_window_mean.argtypes = [_p, C.c_int64, _i, _i, _i, _i, _i, _p, _p]
    L.hops_noise_draw.argtypes = [_p, _i, _p, _i, _i, _i, _p, _p]
    L.hops_noise_seed_states.argtypes = [_p, _p, _i, _p, _p]
    L.hops_noalloc_scratch_bytes.restype = C.c_size_t
    L.hops_noalloc_scratch_bytes.argtypes = [C.POINTER(HopsStructure), _i, _i]
    L.hops_rk4_propagate_noalloc.argtypes = [C.POINTER(HopsStructure), _i, _i, _i, _p, _p, _p,
                                             _i, _p, _i, _i, _i, _i, C.c_double, _p, _p, _p]
    L.hops_stage_tuning.argtypes = [_i, _i]
    L.hops_step_fusion.argtypes = [_i]
    L.hops_grid_barrier_test.argtypes = [_p, _p, _i, _i, _i, C.c_int64, _p]
    L.hops_flux_errors.argtypes = [_p, _i, _i, C.c_double, _p]
    L.hops_tri_max_depth.restype = _i
    L.hops_tri_max_depth.argtypes = []
    L.hops_tri_pass1.argtypes = [_i, _i, _p, C.c_int64, _p, _p, _p, _p]
    L.hops_tri_pass2.argtypes = [_i, _i, _p, C.c_int64, C.c_int64, _p, _p, _p, _p, _p, _p, _p]
    L.hops_batch_settle.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _p]
    L.hops_flux_errors_smem_doubles.restype = _i
    L.hops_flux_errors_smem_doubles.argtypes = [_i, _i, _i]
    L.hops_structure_upload.argtypes = [C.POINTER(HopsStructureDesc), _p, C.POINTER(_p)]
    L.hops_structure_host_view.restype = C.POINTER(HopsStructure)
    L.hops_structure_host_view.argtypes = [_p]
    L.hops_structure_device_view.restype = _p
    L.hops_structure_device_view.argtypes = [_p]
    L.hops_structure_destroy.argtypes = [_p]
    L.hops_batch_create.argtypes = [C.POINTER(HopsStructure), _i, _i, _i,
                                    C.POINTER(C.POINTER(HopsBatch))]
    L.hops_batch_destroy.argtypes = [C.POINTER(HopsBatch)]
    L.hops_batch_set_state_host.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _p,
                                            _p, _p]
    L.hops_batch_set_noise_host.argtypes = [C.POINTER(HopsBatch), _p, _i, _p, _i, _p]
    L.hops_batch_propagate_host.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _i,
                                            _i, _i, C.c_double, _p, _p, _p]
    L.hops_batch_get_state_host.argtypes = [C.POINTER(HopsStructure), C.POINTER(HopsBatch), _p,
                                            _p, _p]
    L.hops_kernel_timing.argtypes = [C.c_int]
    L.hops_kernel_timing_read.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    _lib = L
    return L


def check(rc, what):
    """Map a status code to the reference's exception types."""
    if rc == HOPS_OK:
        return
    msg = lib().hops_last_error().decode(errors="replace")
    if rc == HOPS_ENONFINITE:
        raise TrajectoryError(f"{what}: non-finite state ({msg})")
    if rc == HOPS_ENOTSUP:
        raise UnsupportedRequest(f"{what}: {msg}", what, override=True)
    raise RuntimeError(f"{what} failed with status {rc}: {msg}")


def exported_symbols():
    """Names declared in include/hops_b200.h that the library must export."""
    return ["hops_last_error", "hops_version", "hops_device_query",
            "hops_scalar_workspace_doubles", "hops_batch_reset", "hops_dsystem_dt",
            "hops_rk4_propagate", "hops_resident_propagate", "hops_resident_scalar_doubles",
            "hops_noise_filter", "hops_noise_filter_shared", "hops_noise_filter_work_doubles",
            "hops_kernel_timing",
            "hops_kernel_timing_read", "hops_noalloc_scratch_bytes",
            "hops_rk4_propagate_noalloc", "hops_stage_tuning", "hops_step_fusion",
            "hops_grid_barrier_test",
            "hops_flux_errors",
            "hops_flux_errors_smem_doubles", "hops_tri_max_depth", "hops_tri_pass1",
            "hops_tri_pass2", "hops_noise_window_mean", "hops_noise_draw", "hops_noise_seed_states",
            "hops_batch_settle",
            "hops_structure_upload", "hops_structure_host_view", "hops_structure_device_view",
            "hops_structure_destroy", "hops_batch_create", "hops_batch_destroy",
            "hops_batch_set_state_host", "hops_batch_set_noise_host",
            "hops_batch_propagate_host", "hops_batch_get_state_host"]
