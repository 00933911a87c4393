"""The no-allocation GEMM entry point (phf_ozaki_dgemm_noalloc) against phf_ozaki_dgemm.

Callers that cannot allocate device memory (inside someone else's stream capture, under a
foreign allocator, in loops that must not enter the driver allocator) use the variant whose
scratch lives in a static device array.  It must give the same result as the allocating entry
point, call after call, although every call reuses the same scratch array.  Collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(fn, A, Bt, S):
    import torch

    m, k = A.shape
    n = Bt.shape[0]
    dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(Bt)).cuda()
    dD = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
    st = fn(m, n, k, S, ctypes.c_void_p(dA.data_ptr()), k, ctypes.c_void_p(dB.data_ptr()), k,
            ctypes.c_void_p(dD.data_ptr()), n, ctypes.c_void_p(0))
    _lib.check(st, fn.__name__)
    return dD.cpu().numpy()


def test_noalloc_matches_allocating_entry_two_calls_in_a_row():
    lib = _lib.load()
    rng = np.random.default_rng(123)
    shapes = [(200, 150, 333), (96, 40, 1000)]   # second call: other sizes over the same scratch
    for (m, n, k) in shapes:
        A = rng.normal(size=(m, k)) * 10.0 ** rng.uniform(-2, 2, size=(m, 1))
        Bt = rng.normal(size=(n, k)) * 10.0 ** rng.uniform(-2, 2, size=(n, 1))
        ref = _run(lib.phf_ozaki_dgemm, A, Bt, 6)
        got = _run(lib.phf_ozaki_dgemm_noalloc, A, Bt, 6)
        scale = np.abs(A).max(axis=1)[:, None] * np.abs(Bt).max(axis=1)[None, :]
        # same tolerance as the allocating entry point's own test: (S+1) k 2^-7S per entry, x4
        assert np.all(np.isfinite(got))
        assert (np.abs(got - ref) / scale).max() <= 4.0 * 7 * k * 2.0 ** -42
        assert (np.abs(got - A @ Bt.T) / scale).max() <= 4.0 * 7 * k * 2.0 ** -42


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    need = lib.phf_ozaki_dgemm_noalloc_scratch_bytes(4096, 4096, 4096, 6)
    assert need > 32 << 20
    st = lib.phf_ozaki_dgemm_noalloc(4096, 4096, 4096, 6, ctypes.c_void_p(8), 4096, ctypes.c_void_p(8), 4096,
                                     ctypes.c_void_p(8), 4096, ctypes.c_void_p(0))
    assert st == _lib.PHF_ERR_UNSUPPORTED
    assert b"scratch" in lib.phf_last_error()
