"""The no-allocation GEMM entry point (phf_ozaki_dgemm_noalloc) against phf_ozaki_dgemm.

Callers that cannot allocate device memory (their device memory belongs to another allocator,
or their loops must not enter the driver's allocator) use the variant whose scratch lives in a
static device array.  It must give the same result as the allocating entry point, call after call,
although every call reuses the same scratch array, and after its first calls on a device it must
not change the device's free memory.  Collected last so that a run stopping at the first failure
has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib

pytestmark = pytest.mark.gpu


def _device(A, Bt):
    import torch

    m, n = A.shape[0], Bt.shape[0]
    return (torch.from_numpy(np.ascontiguousarray(A)).cuda(), torch.from_numpy(np.ascontiguousarray(Bt)).cuda(),
            torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda"))


def _call(fn, dA, dB, dD, S, stream=0):
    m, k = dA.shape
    n = dB.shape[0]
    st = fn(m, n, k, S, ctypes.c_void_p(dA.data_ptr()), k, ctypes.c_void_p(dB.data_ptr()), k,
            ctypes.c_void_p(dD.data_ptr()), n, ctypes.c_void_p(stream))
    _lib.check(st, fn.__name__)


def _run(fn, A, Bt, S):
    dA, dB, dD = _device(A, Bt)
    _call(fn, dA, dB, dD, S)
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


def test_noalloc_calls_leave_device_free_memory_unchanged():
    """After the first calls on the device (which load the library's kernels and look up the
    array's address), calls of other sizes must not allocate: the device's free memory, read from
    the driver (cudaMemGetInfo), is the same before and after them.  All tensors of the calls are
    allocated before the first reading, and the calls run on a non-default stream."""
    import torch

    lib = _lib.load()
    rng = np.random.default_rng(7)
    dA, dB, dD = _device(rng.normal(size=(64, 96)), rng.normal(size=(32, 96)))
    for S in (5, 6):  # first calls on this device: every kernel the calls below use is loaded now
        _call(lib.phf_ozaki_dgemm_noalloc, dA, dB, dD, S)
    bufs = [_device(rng.normal(size=(m, k)), rng.normal(size=(n, k))) for m, n, k in
            ((300, 170, 257), (128, 512, 640), (40, 8, 3000))]
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for S in (5, 6):
        for dA2, dB2, dD2 in bufs:
            _call(lib.phf_ozaki_dgemm_noalloc, dA2, dB2, dD2, S, stream.cuda_stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for dA2, dB2, dD2 in bufs:  # and the last products are right
        A, Bt = dA2.cpu().numpy(), dB2.cpu().numpy()
        scale = np.abs(A).max(axis=1)[:, None] * np.abs(Bt).max(axis=1)[None, :]
        k = A.shape[1]
        assert (np.abs(dD2.cpu().numpy() - A @ Bt.T) / scale).max() <= 4.0 * 7 * k * 2.0 ** -42


def test_noalloc_scratch_bytes_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.phf_ozaki_dgemm_noalloc_scratch_bytes(64, 64, 64, 5) > 0
    for args in ((0, 64, 64, 5), (64, -1, 64, 5), (64, 64, 0, 5), (64, 64, 64, 0), (64, 64, 64, 8)):
        assert lib.phf_ozaki_dgemm_noalloc_scratch_bytes(*args) == 0
