"""The floating-point tensor-core precisions (PHF_PREC_BF16X3, PHF_PREC_TF32): the GEMM
phf_tc_dgemm against the CPU emulation of its operand formats, and the energy/gradient pipeline
in those precisions against the FP64 form.

GEMM tolerance: the device result differs from the emulation (converted operands, exact FP64
products) only by FP32 accumulation, bounded by k 2^-23 sum_k |a'||b'| per entry.  At k = 64 /
32 that bound is 30-200x below the effect of a missing cross product or of skipping the TF32
rounding (checked on the CPU), so a wrong layout, quarter or term fails it.  Pipeline: the
relative errors of H, S and the gradient pieces lie in the bands these formats give (BF16x3
about 2^-16, TF32 about 2^-11 per operand), BF16x3 is the closer one, and neither is FP64-exact.
"""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib, api
from tests import _tc_formats as tf

pytestmark = pytest.mark.gpu

PREC = {"bf16x3": 2, "tf32": 3, "ozaki_i8": 1}


def _tc_dgemm(A, Bt, fmt, slices=0):
    import torch

    dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(Bt)).cuda()
    m, k = A.shape
    n = Bt.shape[0]
    dD = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    st = _lib.load().phf_tc_dgemm(m, n, k, PREC[fmt], slices, ctypes.c_void_p(dA.data_ptr()), k,
                                  ctypes.c_void_p(dB.data_ptr()), k, ctypes.c_void_p(dD.data_ptr()), n,
                                  ctypes.c_void_p(0))
    _lib.check(st, "phf_tc_dgemm")
    return dD.cpu().numpy()


@pytest.mark.parametrize("fmt,k", [("bf16x3", 64), ("bf16x3", 40), ("tf32", 32), ("tf32", 20)])
@pytest.mark.parametrize("m,n", [(128, 128), (200, 150), (64, 40)])
def test_tc_dgemm_matches_format_emulation(fmt, k, m, n):
    rng = np.random.default_rng(m + 3 * n + 7 * k + len(fmt))
    A = rng.normal(size=(m, k)) * 10.0 ** rng.uniform(-3, 3, size=(m, 1))
    Bt = rng.normal(size=(n, k)) * 10.0 ** rng.uniform(-3, 3, size=(n, 1))
    D = _tc_dgemm(A, Bt, fmt)
    assert np.isfinite(D).all()
    err = np.abs(D - tf.emulate(A, Bt, fmt)) / tf.accumulation_bound(A, Bt, fmt)
    assert err.max() <= 1.0, err.max()


@pytest.mark.parametrize("fmt,rel", [("bf16x3", 2e-5), ("tf32", 2e-3)])
def test_tc_dgemm_long_k_against_fp64(fmt, rel):
    """k = 3000 runs the operand ring through many laps; the result stays at the format's precision."""
    rng = np.random.default_rng(11)
    A = rng.normal(size=(256, 3000))
    Bt = rng.normal(size=(192, 3000))
    D = _tc_dgemm(A, Bt, fmt)
    ref = A @ Bt.T
    scale = np.abs(A) @ np.abs(Bt).T
    err = np.abs(D - ref) / scale
    assert err.max() <= rel, err.max()
    emu = np.abs(D - tf.emulate(A, Bt, fmt)) / tf.accumulation_bound(A, Bt, fmt)
    assert emu.max() <= 1.0, emu.max()


@pytest.mark.parametrize("fmt,rel", [("bf16x3", 1e-5), ("tf32", 3e-5)])
def test_tc_dgemm_same_sign_sums_keep_the_error_of_one_segment(fmt, rel):
    """Same-sign data with k = 16384 (the exchange GEMM's k at n = 128): the tensor core's FP32
    accumulation rounds towards zero, so one FP32 sum over the whole k range is off by ~1e-4 of the
    result (7.5e-5 for BF16x3, 1.2e-4 for TF32, measured); FP64 sums of 512-element segments keep
    the accumulation error at the level of one segment."""
    rng = np.random.default_rng(13)
    A = np.abs(rng.normal(size=(128, 16384))) + 0.5
    Bt = np.abs(rng.normal(size=(96, 16384))) + 0.5
    D = _tc_dgemm(A, Bt, fmt)
    acc = np.abs(D - tf.emulate(A, Bt, fmt)).max() / np.abs(A @ Bt.T).max()
    assert acc <= rel, acc


def test_tc_dgemm_int8_is_ozaki_dgemm():
    import torch

    rng = np.random.default_rng(12)
    A = rng.normal(size=(130, 77))
    Bt = rng.normal(size=(90, 77))
    D1 = _tc_dgemm(A, Bt, "ozaki_i8", slices=0)
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(Bt).cuda()
    dD = torch.zeros((130, 90), dtype=torch.float64, device="cuda")
    st = _lib.load().phf_ozaki_dgemm(130, 90, 77, 5, ctypes.c_void_p(dA.data_ptr()), 77,
                                     ctypes.c_void_p(dB.data_ptr()), 77, ctypes.c_void_p(dD.data_ptr()), 90,
                                     ctypes.c_void_p(0))
    _lib.check(st, "phf_ozaki_dgemm")
    assert np.array_equal(D1, dD.cpu().numpy())


def test_tc_dgemm_rejects_fp64_precision():
    """The argument check returns before any device memory is touched."""
    lib = _lib.load()
    st = lib.phf_tc_dgemm(8, 8, 8, 0, 0, ctypes.c_void_p(8), 8, ctypes.c_void_p(8), 8, ctypes.c_void_p(8), 8,
                          ctypes.c_void_p(0))
    assert st != 0


def _problem_kwargs(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


@pytest.mark.parametrize("n,N,L", [(60, 21, 50), (72, 10, 40)])
def test_float_precisions_track_fp64_pipeline(n, N, L):
    """n = 60 forms and converts the density columns in one kernel; n = 72 takes the density GEMM
    and the column-conversion kernels."""
    import torch

    from phf_pcc_b200 import synth

    p = synth.make_problem(n, N, L, ngrid=(6, 3), seed=n + N, pg="C2v")
    akw = _problem_kwargs(p)
    C = torch.from_numpy(p.C).cuda()
    res = {}
    for prec in ("fp64", "bf16x3", "tf32"):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, jk_form="eri", precision=prec, **akw) as plan:
            res[prec] = [t.cpu().numpy() for t in plan.eval_device(C)]
    errs = {}
    for prec in ("bf16x3", "tf32"):
        errs[prec] = max(float(np.abs(a - b).max()) / max(1.0, float(np.abs(b).max()))
                         for a, b in zip(res[prec], res["fp64"]))
    assert errs["bf16x3"] <= 1e-4, errs
    assert errs["tf32"] <= 1e-2, errs
    assert 1e-12 < errs["bf16x3"] < errs["tf32"], errs
