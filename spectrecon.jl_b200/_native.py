"""ctypes binding of libspectgpu.so (the C ABI declared in include/spect_gpu.h).

The CUDA library is the only compute path: if it is missing or cannot be
loaded, every entry point raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspectgpu.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_Z = ctypes.c_size_t

class JobDesc(ctypes.Structure):
    """spect_job_desc of include/spect_gpu.h."""

    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("px", ctypes.c_int), ("pz", ctypes.c_int),
                ("nview", ctypes.c_int), ("mumap", ctypes.c_void_p), ("psfs", ctypes.c_void_p),
                ("dy", ctypes.c_float), ("interpmeth", ctypes.c_int), ("ynoisy", ctypes.c_void_p),
                ("background", ctypes.c_void_p), ("x0", ctypes.c_void_p), ("nblocks", ctypes.c_int),
                ("niter", ctypes.c_int)]


_SIGS = {
    "spect_last_error": ([], ctypes.c_char_p),
    "spect_device_info": ([ctypes.POINTER(_I), ctypes.POINTER(_Z)], _I),
    "spect_plan_create": ([ctypes.POINTER(_P), _I, _I, _I, _I, _I, _I, _P, _P, _F, _P, _I, _I, _I, _I], _I),
    "spect_plan_destroy": ([_P], _I),
    "spect_plan_info": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_Z)], _I),
    "spect_plan_conv_kernels": ([_P, ctypes.POINTER(_I)], _I),
    "spect_plan_fused": ([_P, ctypes.POINTER(_I)], _I),
    "spect_plan_fused_taps": ([_P, ctypes.POINTER(ctypes.c_double)], _I),
    "spect_project": ([_P, _P, _P, _P, _I, _P], _I),
    "spect_project_host": ([_P, _P, _P, _P, _I], _I),
    "spect_project_static_scratch": ([_P, _P, _P, _P, _I, _P], _I),
    "spect_backproject": ([_P, _P, _P, _P, _I, _P], _I),
    "spect_backproject_host": ([_P, _P, _P, _P, _I], _I),
    "spect_mlem": ([_P, _P, _P, _P, _P, _I, _P], _I),
    "spect_mlem_host": ([_P, _P, _P, _P, _P, _I], _I),
    "spect_osem": ([_P, _P, _P, _P, _P, _I, _I, _P], _I),
    "spect_osem_host": ([_P, _P, _P, _P, _P, _I, _I], _I),
    "spect_em_subset_update": ([_P, _P, _P, _P, _P, _P, _I, _P], _I),
    "spect_subset_sensitivity": ([_P, _P, _P, _I, _P], _I),
    "spect_plan_autotune": ([_P, _I, _P], _I),
    "spect_batch_create": ([ctypes.POINTER(_P), _I, _P, _P, _P], _I),
    "spect_batch_set_job": ([_P, _I, _P, _P, _P, _P], _I),
    "spect_batch_run": ([_P, _P], _I),
    "spect_batch_destroy": ([_P], _I),
    "spect_server_create": ([ctypes.POINTER(_P), _Z, _I], _I),
    "spect_server_submit": ([_P, ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_longlong)], _I),
    "spect_server_wait": ([_P, ctypes.c_longlong, _P, ctypes.POINTER(ctypes.c_double), _I], _I),
    "spect_server_stats": ([_P, _P], _I),
    "spect_server_destroy": ([_P], _I),
    "spect_kernel_launches": ([], ctypes.c_ulonglong),
    "spect_fp32_peak": ([ctypes.POINTER(_D)], _I),
    "spect_plan_check_error": ([_P, _P], _I),
    "spect_selftest_wait_timeout": ([], _I),
    "spect_plan_profile": ([_P, _I], _I),
    "spect_plan_kernel_times": ([_P, _P, _P], _I),
    "spect_psf_gauss": ([_P, _I, _I, _I, _P, _P], _I),
    "spect_psf_gauss_device": ([_P, _I, _I, _I, _D, _D, _D, _D, _P], _I),
    "spect_plan_create_gauss": ([_P, _I, _I, _I, _I, _I, _I, _P, _D, _D, _D, _D, _F, _P, _I, _I, _I, _I], _I),
}

_lib = None


class SpectError(RuntimeError):
    """A non-zero status from the C ABI; ``code`` is the SPECT_ERR_* value."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """Load libspectgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def symbols():
    return list(_SIGS)


def check(status):
    if status != 0:
        msg = lib().spect_last_error().decode()
        raise SpectError(status, msg)
    return status
