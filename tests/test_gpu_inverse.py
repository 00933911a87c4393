"""The batched overlap inverse (phf_overlap_inverse: InvertC + determinantC of
PHF_fort/Wrappers.f90:195-336) against numpy, through the C ABI.

Sizes cover every kernel form: one warp per matrix (n <= 32), the register-resident elimination
(33..64 and 65..100, two thread-grid shapes with padded rows and columns) and the shared-memory
elimination (101..112).  Matrices where partial pivoting decides the result (zero diagonals, rows
that must be interchanged, exactly tied pivot candidates) are included; an exactly singular matrix
and a non-finite entry are reported with that matrix's outputs zeroed and the others intact.
"""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(S):
    import torch

    batch, n, _ = S.shape
    dS = torch.from_numpy(np.ascontiguousarray(S)).cuda()
    dI = torch.full_like(dS, complex(np.nan, np.nan))
    dd = torch.zeros(batch, dtype=torch.complex128, device="cuda")
    dl = torch.zeros(batch, dtype=torch.complex128, device="cuda")
    df = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = _lib.load()
    st = lib.phf_overlap_inverse(n, batch, ctypes.c_void_p(dS.data_ptr()), ctypes.c_void_p(dI.data_ptr()),
                                 ctypes.c_void_p(dd.data_ptr()), ctypes.c_void_p(dl.data_ptr()),
                                 ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(0))
    return st, dI.cpu().numpy(), dd.cpu().numpy(), dl.cpu().numpy()


def _cases(n, rng):
    """Seeded batch: Gaussian matrices, a permuted upper-triangular one (zero diagonal entries but
    for the interchanges), a near-unitary overlap like C^H R C, and an integer matrix whose pivot
    candidates tie exactly."""
    g = rng.normal(size=(6, n, n)) + 1j * rng.normal(size=(6, n, n))
    perm = rng.permutation(n)
    tri = np.triu(0.2 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))) + 3.0 * np.eye(n)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    ints = (rng.integers(-2, 3, size=(n, n)) + 1j * rng.integers(-2, 3, size=(n, n))) + 4.0 * np.eye(n)
    return np.concatenate([g, tri[perm][None], (q + 1e-3 * g[0])[None], ints[None]])


@pytest.mark.parametrize("n", [7, 32, 33, 48, 64, 65, 77, 100, 101, 112])
def test_inverse_det_logdet_match_numpy(n):
    rng = np.random.default_rng(1000 + n)
    S = _cases(n, rng)
    st, inv, det, logdet = _run(S)
    assert st == _lib.PHF_OK
    for b in range(S.shape[0]):
        ref = np.linalg.inv(S[b])
        cond = np.linalg.cond(S[b])
        scale = np.abs(ref).max()
        # FP64 elimination with partial pivoting: error a modest multiple of cond * eps
        assert np.abs(inv[b] - ref).max() <= 64 * n * cond * 2.0 ** -52 * scale, b
        assert np.abs(inv[b] @ S[b] - np.eye(n)).max() <= 64 * n * cond * 2.0 ** -52, b
        sign, lad = np.linalg.slogdet(S[b])
        assert abs(logdet[b].real - lad) <= 1e-12 * max(1.0, abs(lad)), b
        dphi = np.angle(np.exp(1j * (logdet[b].imag - np.angle(sign))))
        assert abs(dphi) <= 1e-11, b
        assert -np.pi < logdet[b].imag <= np.pi
        assert abs(det[b] - sign * np.exp(lad)) <= 1e-12 * np.exp(lad) * n, b


@pytest.mark.parametrize("n", [20, 40, 100, 110])
def test_singular_and_nonfinite_matrices_are_reported_and_zeroed(n):
    rng = np.random.default_rng(n)
    S = rng.normal(size=(4, n, n)) + 1j * rng.normal(size=(4, n, n))
    S[1][:, n // 2] = 0.0  # exactly singular: a zero column
    st, inv, det, logdet = _run(S)
    assert st == _lib.PHF_ERR_SINGULAR
    assert np.all(inv[1] == 0) and det[1] == 0 and np.isneginf(logdet[1].real)
    for b in (0, 2, 3):
        assert np.abs(inv[b] @ S[b] - np.eye(n)).max() <= 1e-9
    S[1] = S[0]
    S[2][n - 1, 0] = np.nan
    st, inv, det, logdet = _run(S)
    assert st == _lib.PHF_ERR_NONFINITE
    assert np.all(inv[2] == 0) and det[2] == 0
    assert np.abs(inv[3] @ S[3] - np.eye(n)).max() <= 1e-9
