"""ctypes binding of libinqb200 (the C ABI declared in include/inqb200.h).

The library is built in-tree (``inq-wannier-fork_b200/lib/libinqb200.so``).  There
is no fallback: if the library is missing every call raises.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libinqb200.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG), "include", "inqb200.h")

FP64 = 0
MIXED = 1
# theories of the density -> potential step (INQB_THEORY_*)
THEORY_NONE = 0
THEORY_HARTREE = 1
THEORY_LDA = 2
# status of a missing, short or unwritable checkpoint file
ERR_IO = 8
# int (*)(double* rho, long n, void* user): the cross-rank density sum of a sharded SCF step
DENSITY_REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p)

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p
_ctxp = ctypes.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "inqb_version": (ctypes.c_int, []),
    "inqb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "inqb_last_error": (ctypes.c_char_p, []),
    "inqb_grid_supported": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "inqb_ctx_create": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "inqb_ctx_destroy": (ctypes.c_int, [_ctxp]),
    "inqb_ctx_clone": (ctypes.c_int, [_ctxp, ctypes.POINTER(ctypes.c_void_p)]),
    "inqb_ctx_reserve": (ctypes.c_int, [_ctxp, ctypes.c_int]),
    "inqb_volume_element": (ctypes.c_double, [_ctxp]),
    "inqb_cart_to_cov": (ctypes.c_int, [_ctxp, _dp, _dp]),
    "inqb_set_local_potential": (ctypes.c_int, [_ctxp, _dp]),
    "inqb_set_vector_potential": (ctypes.c_int, [_ctxp, _dp]),
    "inqb_set_fourier_sphere_mask": (ctypes.c_int, [_ctxp, ctypes.c_int]),
    "inqb_sphere_size": (ctypes.c_int, [_dp, _ip, _dp, ctypes.c_double, _ip]),
    "inqb_sphere_points": (ctypes.c_int, [_dp, _ip, _dp, ctypes.c_double, ctypes.c_int, _ip, _fp, _fp]),
    "inqb_gaussian_kb_beta": (ctypes.c_int, [_dp, ctypes.c_int, _fp, _fp, ctypes.c_double, _dp]),
    "inqb_set_projectors": (ctypes.c_int, [_ctxp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip, _fp, _dp, _dp]),
    "inqb_apply_h": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_apply_h_host": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int]),
    "inqb_fft_forward": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_fft_backward": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_exponential": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, _vp]),
    "inqb_etrs_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _vp]),
    "inqb_density": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "inqb_dipole": (ctypes.c_int, [_ctxp, _vp, _dp, _vp]),
    "inqb_orthonormalize": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_band_energies": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, _dp, _vp]),
    "inqb_orthonormalize_noalloc": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_set_projection_mode": (ctypes.c_int, [_ctxp, ctypes.c_int]),
    "inqb_device_status": (ctypes.c_int, [_ctxp, _vp]),
    "inqb_timing_passes": (ctypes.c_int, [_ctxp, _dp, _ip]),
    "inqb_mlwf_gram_block": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                            _vp, _vp]),
    "inqb_mlwf_finish": (ctypes.c_int, [_ctxp, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "inqb_orbital_norms": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "inqb_mlwf_centres": (ctypes.c_int, [_ctxp, ctypes.c_int, _dp, _dp, _dp]),
    "inqb_overlap_block": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                          _vp, ctypes.c_int, _vp]),
    "inqb_cholesky_inverse": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_rotate_block": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                         _vp, ctypes.c_int, _vp]),
    "inqb_autotune": (ctypes.c_int, [_ctxp, ctypes.c_int, _vp, _ip]),
    "inqb_set_schedule": (ctypes.c_int, [_ctxp, ctypes.c_int, _ip]),
    "inqb_crank_nicolson_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                                ctypes.c_int, ctypes.c_double, _ip, _dp, _vp]),
    "inqb_kick": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _dp, _vp]),
    "inqb_poisson": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "inqb_ks_potential": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, _dp, _vp]),
    "inqb_etrs_scf_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _vp,
                                          _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip, _dp, _vp]),
    "inqb_crank_nicolson_scf_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp,
                                                    _dp, _vp, ctypes.c_double, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_double, _ip, _dp, _dp, _vp]),
    "inqb_save_orbitals": (ctypes.c_int, [_ctxp, ctypes.c_char_p, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _dp, _vp]),
    "inqb_load_orbitals": (ctypes.c_int, [_ctxp, ctypes.c_char_p, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _dp, _vp]),
    "inqb_save_density": (ctypes.c_int, [_ctxp, ctypes.c_char_p, _vp, _vp]),
    "inqb_load_density": (ctypes.c_int, [_ctxp, ctypes.c_char_p, _vp, _vp]),
    "inqb_mlwf_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip,
                                      _dp, _dp, _vp]),
    "inqb_mlwf_matrices": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "inqb_jade": (ctypes.c_int, [_ctxp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double, _ip, _vp]),
    "inqb_mlwf_rotate": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "inqb_set_density_reduce": (ctypes.c_int, [_ctxp, _vp, _vp]),
    "inqb_etrs_powers_size": (ctypes.c_int, [_ctxp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "inqb_etrs_step_powers": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                             _vp, _vp]),
    "inqb_etrs_step_terms": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                            _vp]),
    "inqb_etrs_adjoint_step": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                              _vp, _vp, _vp, _vp, _vp]),
    "inqb_axpby": (ctypes.c_int, [_ctxp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, _vp, ctypes.c_int, _vp]),
    "inqb_position_scale": (ctypes.c_int, [_ctxp, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           _vp, ctypes.c_double, _vp]),
    "inqb_accum_potential_gradient": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                     ctypes.c_double, _vp, _vp]),
    "inqb_accum_vector_potential_gradient": (ctypes.c_int, [_ctxp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                                            ctypes.c_double, ctypes.c_double, _vp, _vp]),
    "inqb_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "inqb_batch_destroy": (ctypes.c_int, [_vp]),
    "inqb_batch_apply_h": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), _ip,
                                          _ip, _vp]),
    "inqb_batch_set_mode": (ctypes.c_int, [_vp, ctypes.c_int]),
    "inqb_batch_autotune": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                           _ip, _ip, _vp, _ip, _dp]),
    "inqb_batch_info": (ctypes.c_int, [_vp, _ip, _ip, _ip]),
    "inqb_batch_status": (ctypes.c_int, [_vp, _vp]),
    "inqb_batch_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_double]),
    "inqb_batch_test_unreachable_wait": (ctypes.c_int, [_vp, ctypes.c_int]),
    "inqb_timing_start": (ctypes.c_int, [_ctxp, ctypes.c_int]),
    "inqb_timing_stop": (ctypes.c_int, [_ctxp, _dp, _ip]),
}

_lib = None


class InqbError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


def lib():
    """Load libinqb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libinqb200.so not built: run `python inq-wannier-fork_b200/build.py` ({LIB_PATH})")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != 0:
        msg = lib().inqb_last_error().decode(errors="replace")
        raise InqbError(status, where, msg)


def call(name: str, *args):
    """Call a status-returning entry point and raise on failure."""
    check(getattr(lib(), name)(*args), name)


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def fptr(a):
    return a.ctypes.data_as(_fp)
