"""ctypes binding of libvox.so (include/vox.h).

The library is loaded from this package directory only; if it is missing the
import fails loudly - there is no CPU fallback for the hot path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvox.so")

VOX_OK = 0
VOX_ERR_BAD_ARG = 1
VOX_ERR_OOM = 2
VOX_ERR_NOT_CONVERGED = 3
VOX_ERR_TIMEOUT = 4
VOX_ERR_CUDA = 5
VOX_ERR_UNSUPPORTED = 6

VOX_C128 = 0
VOX_C64 = 1
PREC = {"c128": VOX_C128, "c64": VOX_C64, "double": VOX_C128, "single": VOX_C64}
SIDE = {None: 0, "none": 0, "L": 1, "left": 1, "R": 2, "right": 2}

_dp = ctypes.POINTER(ctypes.c_double)


class VoxError(RuntimeError):
    """A libvox call returned a non-OK vox_status."""

    def __init__(self, status, msg):
        super().__init__(f"libvox status {status}: {msg}")
        self.status = status


class OpDesc(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_int), ("M", ctypes.c_int), ("N", ctypes.c_int),
        ("LfN", ctypes.c_int), ("MfN", ctypes.c_int), ("NfN", ctypes.c_int),
        ("fN_re", _dp), ("fN_im", _dp),
        ("G_re", _dp), ("G_im", _dp),
        ("Mr_re", _dp), ("Mr_im", _dp),
        ("Mc_re", _dp), ("Mc_im", _dp),
        ("gram", ctypes.c_double),
        ("idx", _dp), ("n_idx", ctypes.c_longlong),
        ("precisions", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class GmresInfo(ctypes.Structure):
    _fields_ = [
        ("flag", ctypes.c_int),
        ("relres", ctypes.c_double),
        ("iter_inner", ctypes.c_int),
        ("iter_outer", ctypes.c_int),
        ("total_iters", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("resvec", _dp),
        ("resvec_cap", ctypes.c_longlong),
        ("n_resvec", ctypes.c_longlong),
        ("seconds", ctypes.c_double),
    ]


class JvieDesc(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_int), ("M", ctypes.c_int), ("N", ctypes.c_int),
        ("Einc_re", _dp), ("Einc_im", _dp),
        ("er_re", _dp), ("er_im", _dp),
        ("dx", ctypes.c_double), ("freq", ctypes.c_double),
        ("LfN", ctypes.c_int), ("MfN", ctypes.c_int), ("NfN", ctypes.c_int),
        ("fN_re", _dp), ("fN_im", _dp),
        ("G_re", _dp), ("G_im", _dp),
        ("tol", ctypes.c_double),
        ("form", ctypes.c_int),
        ("solver", ctypes.c_char),
        ("precond", ctypes.c_char),
        ("inner_it", ctypes.c_int),
        ("outer_it", ctypes.c_int),
        ("prec", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


# (name, restype, argtypes) for every entry point declared in include/vox.h
SIGNATURES = [
    ("vox_last_error", ctypes.c_char_p, []),
    ("vox_abi_version", ctypes.c_int, []),
    ("vox_set_wait_timeout", ctypes.c_int, [ctypes.c_double]),
    ("vox_get_wait_timeout", ctypes.c_double, []),
    ("vox_mem_in_use", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    ("vox_jvie_solve", ctypes.c_int, [ctypes.POINTER(JvieDesc), _dp, _dp,
                                      ctypes.POINTER(GmresInfo)]),
    ("vox_op_create", ctypes.c_int, [ctypes.POINTER(OpDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_op_destroy", None, [ctypes.c_void_p]),
    ("vox_op_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_longlong)]),
    ("vox_mv_AN", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("vox_mv_L", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("vox_mv_AN_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vox_mv_AN_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("vox_precond_apply_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    ("vox_mv_AN_batch_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    ("vox_block_dot", ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                     ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p]),
    ("vox_block_update", ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                        ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong,
                                        ctypes.c_void_p]),
    ("vox_precond_create_level1", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp,
                                                 ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_precond_create_blocks", ctypes.c_int, [ctypes.c_void_p, _dp, _dp,
                                                 ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_precond_destroy", None, [ctypes.c_void_p]),
    ("vox_precond_apply", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("vox_pgmres", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp,
                                  ctypes.POINTER(GmresInfo)]),
    ("vox_solve_refined", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _dp, _dp,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, _dp, _dp,
                                         ctypes.POINTER(GmresInfo)]),
    ("vox_pgmres_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.POINTER(GmresInfo)]),
    ("vox_solve_refined_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.POINTER(GmresInfo)]),
    ("vox_jvie_rhs", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp,
                                    ctypes.c_double, ctypes.c_double, _dp, ctypes.c_longlong,
                                    _dp, _dp]),
    ("vox_assemble_toeplitz", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             _dp, _dp]),
    ("vox_assemble_toeplitz_device", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_int, _dp, _dp]),
    ("vox_singular_integrals", ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              _dp]),
    ("vox_op_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("vox_op_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    ("vox_op_flags", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("vox_op_interp", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), _dp,
                                     ctypes.c_int]),
    ("vox_precond_share", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_precond_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]),
    ("vox_profile_stages", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]),
    ("vox_op_create_batch", ctypes.c_int, [ctypes.POINTER(OpDesc), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_op_members", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("vox_op_interp_member", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p), _dp, ctypes.c_int]),
    ("vox_solve_refined_batch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_int, _dp, _dp, ctypes.c_double,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_int, _dp, _dp,
                                               ctypes.POINTER(GmresInfo)]),
    ("vox_precond_create_box", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_void_p, _dp, _dp, _dp, _dp,
                                              ctypes.c_double, ctypes.c_double,
                                              ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_precond_create_sum", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_lane_create", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    ("vox_lane_destroy", None, [ctypes.c_void_p]),
    ("vox_lane_submit_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    ("vox_lane_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp]),
    ("vox_lane_step", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]),
    ("vox_lane_collect", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp,
                                        ctypes.POINTER(GmresInfo)]),
    ("vox_lane_state", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("vox_solve_refined_batch_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                      ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_void_p, ctypes.c_double,
                                                      ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_double, ctypes.c_int,
                                                      ctypes.c_void_p,
                                                      ctypes.POINTER(GmresInfo)]),
]

_LIB = None


def lib():
    """Load libvox.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python -m voxphoton_b200.build` "
                "(the CUDA library is required; there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(status):
    if status != VOX_OK:
        msg = lib().vox_last_error()
        raise VoxError(status, msg.decode() if msg else "")


def mem_in_use(device=0):
    """Device bytes libvox holds on `device` (vox_mem_in_use)."""
    b = ctypes.c_longlong(0)
    check(lib().vox_mem_in_use(int(device), ctypes.byref(b)))
    return int(b.value)


def dptr(a):
    """Pointer to a C-contiguous float64 array, or NULL for None."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def split(z, n=None):
    """complex array -> (re, im) contiguous float64 (MATLAB split storage)."""
    z = np.asarray(z)
    re = np.ascontiguousarray(np.real(z), dtype=np.float64).reshape(-1)
    im = np.ascontiguousarray(np.imag(z), dtype=np.float64).reshape(-1)
    if n is not None and re.size != n:
        raise ValueError(f"expected {n} entries, got {re.size}")
    return re, im


def fortran_flat(a):
    """MATLAB column-major flattening."""
    return np.asarray(a).reshape(-1, order="F")
