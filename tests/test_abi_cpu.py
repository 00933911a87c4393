"""The C ABI library without a GPU: it loads, exports every declared symbol, and fails loudly."""
import os
import re

import numpy as np
import pytest

from phf_pcc_b200 import _lib, api
from phf_pcc_b200.PHFTools_F import phftools

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(phf_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert "phf_buildhsg" in names and "phf_localg" in names
    for name in names:
        assert hasattr(lib, name), name
    # the ctypes signature table covers every declared entry point
    assert set(names) <= set(_lib.SIGNATURES)


def test_version_and_status_strings():
    lib = _lib.load()
    assert lib.phf_version().startswith(b"phf_b200")
    assert lib.phf_status_string(_lib.PHF_ERR_SINGULAR) == b"singular rotated overlap"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_no_device_raises_instead_of_cpu_fallback():
    with pytest.raises(_lib.PHFError) as ei:
        api.localg(np.zeros((1, 1, 4, 4)), np.zeros((1, 1, 4, 4)), np.ones((1, 1)), 1.0, [1.0], [1.0], [1.0], 1)
    assert ei.value.status == _lib.PHF_ERR_NO_DEVICE


def test_shim_checks_shapes_before_calling_the_library():
    M, N = 6, 2
    eye = np.eye(M, dtype=complex)[None]
    with pytest.raises(ValueError):
        phftools.buildhsg(np.eye(M), np.zeros((M, M, M, M)), np.eye(M), np.zeros((M - N, N)), [1, 1], 1, 1, 1, N,
                          eye, eye, eye, np.ones((1, 2)), np.ones((1, 1, 1)), [0.0], [0.0], [0.0], 0, 1, 0)
    with pytest.raises(ValueError):  # wrong z shape
        phftools.buildhsg(np.eye(M), np.zeros((M, M, M, M)), np.eye(M), np.zeros((M, N)), [1, 1], 1, 1, 1, N,
                          eye, eye, eye, np.ones((1, 1)), np.ones((1, 1, 1)), [0.0], [0.0], [0.0], 0, 1, 0)


def test_tensor_core_gemm_entries_validate_arguments_before_any_device_call():
    """phf_tc_dgemm and phf_ozaki_dgemm reject bad precisions, slice counts and sizes with
    PHF_ERR_ARG before touching device memory (the pointers here are never dereferenced)."""
    import ctypes

    lib = _lib.load()
    p = ctypes.c_void_p(8)
    null = ctypes.c_void_p(0)
    # precision FP64 (0) and unknown (7) are not tensor-core precisions
    for prec in (0, 7):
        assert lib.phf_tc_dgemm(8, 8, 8, prec, 0, p, 8, p, 8, p, 8, null) == _lib.PHF_ERR_ARG
    # int8 slice counts outside 0..7
    for slices in (-1, 8):
        assert lib.phf_tc_dgemm(8, 8, 8, 1, slices, p, 8, p, 8, p, 8, null) == _lib.PHF_ERR_ARG
    assert lib.phf_ozaki_dgemm(8, 8, 8, 0, p, 8, p, 8, p, 8, null) == _lib.PHF_ERR_ARG
    # leading dimensions below the row length, empty sizes, null operands
    assert lib.phf_tc_dgemm(8, 8, 8, 2, 0, p, 4, p, 8, p, 8, null) == _lib.PHF_ERR_ARG
    assert lib.phf_tc_dgemm(0, 8, 8, 3, 0, p, 8, p, 8, p, 8, null) == _lib.PHF_ERR_ARG
    assert lib.phf_tc_dgemm(8, 8, 8, 2, 0, null, 8, p, 8, p, 8, null) == _lib.PHF_ERR_ARG


def test_overlap_inverse_validates_arguments_before_any_device_call():
    """phf_overlap_inverse rejects empty sizes and null pointers (PHF_ERR_ARG) and n above the
    inverse's limit of 112 (PHF_ERR_UNSUPPORTED) before touching device memory."""
    import ctypes

    lib = _lib.load()
    p = ctypes.c_void_p(8)
    null = ctypes.c_void_p(0)
    assert lib.phf_overlap_inverse(0, 4, p, p, p, p, p, null) == _lib.PHF_ERR_ARG
    assert lib.phf_overlap_inverse(8, 0, p, p, p, p, p, null) == _lib.PHF_ERR_ARG
    assert lib.phf_overlap_inverse(8, 4, p, p, p, p, null, null) == _lib.PHF_ERR_ARG
    assert lib.phf_overlap_inverse(113, 4, p, p, p, p, p, null) == _lib.PHF_ERR_UNSUPPORTED


def test_pbarhbarolap_rejects_options_before_any_device_call():
    """TrunODE outside 1..3 is an error (the reference STOPs) and nso above the inverse's limit is
    refused -- both before device memory is touched."""
    import ctypes

    lib = _lib.load()
    p = ctypes.c_void_p(8)
    ng = (ctypes.c_int * 2)(1, 1)

    def call(nocc=2, nso=8, trunode=1, ncisp=1, qj=0, ncik=1):
        return lib.phf_pbarhbarolap(p, p, p, p, p, p, p, p, p, p, p, nocc, nso // 2, nso, 0.0, qj, 1, ng, 1, ncisp, 1,
                                    ncik, p, p, p, p, p, p, p, p, p, p, p, p, trunode, 0)

    assert call(trunode=0) == _lib.PHF_ERR_ARG
    assert call(trunode=-4) == _lib.PHF_ERR_ARG
    assert call(trunode=4) == _lib.PHF_ERR_ARG
    assert call(nso=114, nocc=4) == _lib.PHF_ERR_UNSUPPORTED
    assert call(ncisp=2) == _lib.PHF_ERR_ARG      # ncisp must be 2 qj + 1
    assert call(ncik=3) == _lib.PHF_ERR_ARG
    assert call(nocc=8) == _lib.PHF_ERR_ARG        # no virtual orbitals


def test_plan_rejects_exchange_options_before_any_device_call():
    """exchange_symmetry outside 0..2 and a negative exchange_panel are argument errors of
    phf_plan_create, found before the device is touched (the pointers are never dereferenced)."""
    import ctypes

    lib = _lib.load()
    ng = (ctypes.c_int * 2)(1, 1)

    def create(**kw):
        d = _lib.phf_plan_desc()
        d.nso, d.nocc, d.nchol, d.npg, d.nci, d.ncisp, d.ncipg, d.cmplxconj, d.sp = 8, 2, 3, 1, 1, 1, 1, 1, 1
        d.ngrid = ctypes.cast(ng, ctypes.c_void_p)
        for f in ("h", "bvec", "ref", "r1", "r2", "rpg", "weightsp", "weightpg", "roota", "rootb", "rooty"):
            setattr(d, f, 8)
        d.jk_form = 3
        for k, v in kw.items():
            setattr(d, k, v)
        h = ctypes.c_void_p()
        return lib.phf_plan_create(ctypes.byref(d), ctypes.byref(h))

    assert create(exchange_symmetry=3) == _lib.PHF_ERR_ARG
    assert b"exchange_symmetry" in lib.phf_last_error()
    assert create(exchange_symmetry=-1) == _lib.PHF_ERR_ARG
    assert create(exchange_panel=-1) == _lib.PHF_ERR_ARG


def test_comparison_settings_round_trip_without_a_device():
    """phf_int8_fock_product and phf_int8_wide_mma only set host-side flags that plans read when they
    are created: each returns the previous value, and values above 1 of the first (a sub-batch cap)
    are kept as given."""
    lib = _lib.load()
    was_fx, was_wide = lib.phf_int8_fock_product(0), lib.phf_int8_wide_mma(1)
    try:
        assert lib.phf_int8_fock_product(1) == 0
        assert lib.phf_int8_fock_product(7) == 1
        assert lib.phf_int8_fock_product(-3) == 7  # negative: off
        assert lib.phf_int8_fock_product(1) == 0
        assert lib.phf_int8_wide_mma(0) == 1
        assert lib.phf_int8_wide_mma(1) == 0
    finally:
        lib.phf_int8_fock_product(was_fx)
        lib.phf_int8_wide_mma(was_wide)
