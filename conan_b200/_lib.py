"""ctypes binding of libconan_pm.so (declarations mirror include/conan_pm.h).

The library must have been built in-tree (``python conan_b200/build.py``);
importing this module fails loudly when it is missing -- there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libconan_pm.so"

OK, ERR_ARG, ERR_ALLOC, ERR_CUDA, ERR_TIMEOUT, ERR_IO, ERR_STATE, ERR_UNSUPPORTED = range(8)
FP32, FP64 = 0, 1
GRAD_FD4, GRAD_SPECTRAL = 0, 1
DEPOSIT_SORTED, DEPOSIT_LAGRANGIAN = 0, 1

_dp = C.POINTER(C.c_double)


class ICParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("mbits", C.c_int), ("size", C.c_double), ("seed", C.c_ulong),
                ("ns", C.c_double), ("smooth", C.c_int), ("scale_free", C.c_int), ("scale", C.c_double),
                ("sigma", C.c_double), ("Omega0", C.c_double), ("H0", C.c_double),
                ("precision", C.c_int), ("device", C.c_int)]


class PMParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_mass", C.c_int), ("f", C.c_int), ("size", C.c_double),
                ("H0", C.c_double), ("Omega_m", C.c_double), ("Omega_L", C.c_double),
                ("precision", C.c_int), ("gradient", C.c_int), ("periodic_gather", C.c_int),
                ("device", C.c_int)]


class CicParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_mass", C.c_int), ("f", C.c_int), ("size", C.c_double),
                ("sub_sample", C.c_int), ("device", C.c_int)]


class FofParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_particles", C.c_ulonglong), ("size", C.c_double),
                ("linking_length", C.c_double), ("device", C.c_int)]


class DiffParams(C.Structure):
    _fields_ = [("ic", ICParams), ("pm", PMParams), ("a0", C.c_double), ("da", C.c_double),
                ("n", C.c_uint), ("checkpoint_every", C.c_uint)]


class EnsMember(C.Structure):
    _fields_ = [("mbits", C.c_int), ("size", C.c_double), ("ns", C.c_double), ("seed", C.c_ulong)]


class EnsParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("H0", C.c_double), ("Omega_m", C.c_double), ("Omega_L", C.c_double),
                ("sigma", C.c_double), ("scale", C.c_double), ("a0", C.c_double), ("da", C.c_double),
                ("n", C.c_uint), ("precision", C.c_int), ("device", C.c_int), ("autotune", C.c_int)]


STEP_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint, C.c_double, C.c_void_p)

# name -> (restype, argtypes); every symbol declared in include/conan_pm.h.
SIGNATURES = {
    "conan_last_error": (C.c_char_p, []),
    "conan_version": (C.c_char_p, []),
    "conan_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "conan_selftest_bounded_wait": (C.c_int, [C.c_uint, C.c_void_p]),
    "conan_ic_noise": (C.c_int, [C.POINTER(ICParams), _dp]),
    "conan_ic_generate": (C.c_int, [C.POINTER(ICParams), _dp, _dp]),
    "conan_ic_potential": (C.c_int, [C.POINTER(ICParams), _dp]),
    "conan_ic_displacement": (C.c_int, [C.POINTER(ICParams), _dp, _dp]),
    "conan_cic": (C.c_int, [C.POINTER(CicParams), _dp, _dp]),
    "conan_fof": (C.c_int, [C.POINTER(FofParams), _dp, C.c_void_p, C.POINTER(C.c_ulonglong)]),
    "conan_fof_create": (C.c_void_p, [C.POINTER(FofParams)]),
    "conan_fof_destroy": (None, [C.c_void_p]),
    "conan_fof_run": (C.c_int, [C.c_void_p, _dp, C.c_void_p, C.POINTER(C.c_ulonglong)]),
    "conan_fof_run_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_ulonglong),
                                       C.c_void_p]),
    "conan_pm_create": (C.c_void_p, [C.POINTER(PMParams)]),
    "conan_pm_destroy": (None, [C.c_void_p]),
    "conan_pm_init": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double]),
    "conan_pm_drift": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "conan_pm_kick": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "conan_pm_set_callback_interval": (C.c_int, [C.c_void_p, C.c_uint]),
    "conan_pm_set_deposit": (C.c_int, [C.c_void_p, C.c_int]),
    "conan_pm_get_deposit": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "conan_pm_run": (C.c_int, [C.c_void_p, _dp, C.c_double, C.c_double, C.c_uint, STEP_CB, C.c_void_p]),
    "conan_pm_get_state": (C.c_int, [C.c_void_p, _dp, _dp]),
    "conan_pm_set_state": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double, C.c_double]),
    "conan_pm_scale_factors": (C.c_int, [C.c_void_p, _dp, _dp]),
    "conan_pm_density": (C.c_int, [C.c_void_p, _dp]),
    "conan_pm_potential": (C.c_int, [C.c_void_p, _dp]),
    "conan_pm_power_spectrum": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    "conan_pm_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "conan_pm_profile_entry": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.POINTER(C.c_int), _dp]),
    "conan_pm_profile_reset": (C.c_int, [C.c_void_p]),
    "conan_pm_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "conan_pm_sync": (C.c_int, [C.c_void_p]),
    "conan_pm_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "conan_pm_autotune": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_char_p, C.c_size_t]),
    "conan_diff_create": (C.c_void_p, [C.POINTER(DiffParams)]),
    "conan_diff_destroy": (None, [C.c_void_p]),
    "conan_diff_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "conan_diff_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "conan_ens_create": (C.c_void_p, [C.POINTER(EnsParams), C.c_int, C.POINTER(EnsMember)]),
    "conan_ens_destroy": (None, [C.c_void_p]),
    "conan_ens_init": (C.c_int, [C.c_void_p]),
    "conan_ens_run": (C.c_int, [C.c_void_p]),
    "conan_ens_forward_adjoint": (C.c_int, [C.c_void_p, _dp]),
    "conan_ens_power_spectrum": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp]),
    "conan_ens_state": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "conan_ens_member_fields": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    "conan_ens_last_ms": (C.c_int, [C.c_void_p, _dp, _dp]),
    "conan_ens_total_particles": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "conan_ens_describe": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "conan_deposit_static": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
}


class ConanError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[conan error {code}] {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded library (declared signatures); raises if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python conan_b200/build.py`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().conan_last_error().decode()


def check(rc: int):
    if rc != OK:
        raise ConanError(rc, last_error())


def ptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)
