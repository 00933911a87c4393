"""ctypes binding of libphf_b200.so (the C ABI declared in include/phf_b200.h).

The shared library is the only compute path: if it is missing or no CUDA device is
present, calls raise instead of falling back to a CPU implementation."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphf_b200.so")

PHF_OK = 0
PHF_ERR_ARG = 1
PHF_ERR_SINGULAR = 2
PHF_ERR_NOT_HERMITIAN = 3
PHF_ERR_NONFINITE = 4
PHF_ERR_CUDA = 5
PHF_ERR_OOM = 6
PHF_ERR_UNSUPPORTED = 7
PHF_ERR_NO_DEVICE = 8

PREC = {"fp64": 0, "ozaki_i8": 1, "bf16x3": 2, "tf32": 3}


class phf_complex(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]


class phf_plan_desc(ctypes.Structure):
    _fields_ = [
        ("nso", ctypes.c_int), ("nocc", ctypes.c_int), ("nchol", ctypes.c_int),
        ("h", ctypes.c_void_p), ("bvec", ctypes.c_void_p),
        ("hone", ctypes.c_void_p), ("htwo", ctypes.c_void_p),
        ("ref", ctypes.c_void_p),
        ("ngrid", ctypes.c_void_p),
        ("npg", ctypes.c_int), ("nci", ctypes.c_int), ("ncisp", ctypes.c_int), ("ncipg", ctypes.c_int),
        ("cmplxconj", ctypes.c_int), ("qj", ctypes.c_int), ("sp", ctypes.c_int),
        ("r1", ctypes.c_void_p), ("r2", ctypes.c_void_p), ("rpg", ctypes.c_void_p),
        ("weightsp", ctypes.c_void_p), ("weightpg", ctypes.c_void_p), ("roota", ctypes.c_void_p),
        ("rootb", ctypes.c_void_p), ("rooty", ctypes.c_void_p),
        ("precision", ctypes.c_int), ("slices", ctypes.c_int),
        ("workspace_bytes", ctypes.c_size_t),
        ("jk_form", ctypes.c_int),
        ("gradient_mode", ctypes.c_int),
        ("fp64_library_gemm", ctypes.c_int),
        ("point_begin", ctypes.c_int),
        ("point_end", ctypes.c_int),
        ("exchange_panel", ctypes.c_int),
        ("autotune", ctypes.c_int),
        ("exchange_symmetry", ctypes.c_int),
    ]


# Every symbol include/phf_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
SIGNATURES = {
    "phf_buildhsg": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I,
                          _P, _P, _P, _P]),
    "phf_buildhsg_chol": (_I, [_P, _P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P,
                               _I, _I, _I, _P, _P, _P, _P]),
    "phf_localg": (_I, [_P, _P, _P, phf_complex, _I, _P, _P, _P, _I, _I, _I, _I, _P]),
    "phf_plan_create": (_I, [ctypes.POINTER(phf_plan_desc), ctypes.POINTER(_P)]),
    "phf_plan_destroy": (_I, [_P]),
    "phf_plan_buildhsg": (_I, [_P, _P, _P, _P, _P, _P]),
    "phf_plan_eval_device": (_I, [_P, _P, _P, _P, _P, _P]),
    "phf_plan_eval_device_async": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "phf_eval_batch": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "phf_batch_branches": (_I, []),
    "phf_plan_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_size_t)]),
    "phf_status_string": (ctypes.c_char_p, [_I]),
    "phf_last_error": (ctypes.c_char_p, []),
    "phf_kernel_launches": (ctypes.c_ulonglong, []),
    "phf_version": (ctypes.c_char_p, []),
    "phf_tuned_shapes": (_I, []),
    "phf_int8_wide_mma": (_I, [_I]),
    "phf_int8_fock_product": (_I, [_I]),
    "phf_buildsc": (_I, [phf_complex, _P, _P, _I, _I, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                         _P, _P, _P, _P, _P]),
    "phf_pbarhbarolap": (_I, [_P] * 11 + [_I, _I, _I, ctypes.c_double, _I, _I, _P, _I, _I, _I, _I] + [_P] * 12
                         + [_I, ctypes.c_size_t]),
    "phf_pbarhbarolap_stats": (_I, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "phf_profile_enable": (_I, [_I]),
    "phf_ozaki_dgemm": (_I, [_I, _I, _I, _I, _P, ctypes.c_longlong, _P, ctypes.c_longlong, _P, ctypes.c_longlong, _P]),
    "phf_tc_dgemm": (_I, [_I, _I, _I, _I, _I, _P, ctypes.c_longlong, _P, ctypes.c_longlong, _P, ctypes.c_longlong,
                          _P]),
    "phf_ozaki_dgemm_noalloc": (_I, [_I, _I, _I, _I, _P, ctypes.c_longlong, _P, ctypes.c_longlong, _P,
                                     ctypes.c_longlong, _P]),
    "phf_ozaki_dgemm_noalloc_scratch_bytes": (ctypes.c_size_t, [_I, _I, _I, _I]),
    "phf_overlap_inverse": (_I, [_I, _I, _P, _P, _P, _P, _P, _P]),
    "phf_profile_read": (_I, [_I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_ulonglong)]),
}

_lib = None


class PHFError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def load(path: str = LIB_PATH):
    """Load the CUDA library (building it first only if the sources are present and it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m phf_pcc_b200.build` "
                          "(there is no CPU implementation to fall back to)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str = "phf call"):
    if status == PHF_OK:
        return
    lib = load()
    msg = lib.phf_last_error().decode(errors="replace")
    name = lib.phf_status_string(status).decode()
    raise PHFError(status, f"{what}: {name}" + (f" ({msg})" if msg else ""))


def kernel_launches() -> int:
    return int(load().phf_kernel_launches())


PROF_JK, PROF_GEMM, PROF_INVERSE, PROF_MEMORY = 0, 1, 2, 3


def profile_enable(on: bool = True):
    load().phf_profile_enable(1 if on else 0)


def profile_read(cls: int):
    """(total device milliseconds, launch count) of kernel class ``cls`` since profile_enable."""
    ms = ctypes.c_double()
    n = ctypes.c_ulonglong()
    load().phf_profile_read(cls, ctypes.byref(ms), ctypes.byref(n))
    return float(ms.value), int(n.value)
