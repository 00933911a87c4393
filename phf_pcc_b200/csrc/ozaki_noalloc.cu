// FP64-accurate int8 GEMM for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc at the point where they need a product:
// applications whose device-memory pool is owned by another allocator (a framework caching
// allocator, a fixed arena set up at start, where an allocation of this library's own would
// fail or split the pool), and latency-critical loops that must not enter the driver's
// allocator (cudaMalloc and cudaFree can synchronize the device).  phf_ozaki_dgemm_noalloc
// computes the same product as phf_ozaki_dgemm but keeps
// its scratch (the int8 slices of both operands, their power-of-two exponents and the
// pipeline error flag) in one file-scope device array of kNoAllocScratchBytes, which every
// GPU that loads this library holds until the process exits.  The caller still provides A, B
// and D.  Sizes whose scratch does not fit are rejected with PHF_ERR_UNSUPPORTED.
//
// All calls share the one array and it keeps the contents of the last call: the parts that
// must start at zero (slice padding, the error flag) are cleared on every call, and calls
// that overlap on the GPU (different streams, or different host threads on one device)
// race on it.  The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that first call
// before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "phf_internal.h"

namespace phf {
namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;  // 32 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[kMaxDevices] = {};

int scratch_address(unsigned char **out) {
    int dev = 0;
    PHF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(PHF_ERR_UNSUPPORTED, "phf_ozaki_dgemm_noalloc: device ordinal out of range");
        return PHF_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(PHF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            return PHF_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = reinterpret_cast<unsigned char *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return PHF_OK;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace phf

extern "C" size_t phf_ozaki_dgemm_noalloc_scratch_bytes(int m, int n, int k, int slices) {
    using namespace phf;
    if (m <= 0 || n <= 0 || k <= 0 || slices < 1 || slices > 7) return 0;
    const long long mp = oz_pad_rows(m), np = oz_pad_cols(n);
    return align256(oz_slice_bytes(mp, k, slices)) + align256(oz_slice_bytes(np, k, slices)) + align256(mp * sizeof(int)) +
           align256(np * sizeof(int)) + align256(sizeof(int));
}

extern "C" int phf_ozaki_dgemm_noalloc(int m, int n, int k, int slices, const double *dA, long long lda,
                                       const double *dBt, long long ldb, double *dD, long long ldd, void *stream) {
    using namespace phf;
    set_error(PHF_OK, "");
    if (m <= 0 || n <= 0 || k <= 0 || !dA || !dBt || !dD || lda < k || ldb < k || ldd < n || slices < 1 ||
        slices > 7) {
        set_error(PHF_ERR_ARG, "phf_ozaki_dgemm_noalloc: bad sizes, slices or null pointer");
        return PHF_ERR_ARG;
    }
    const size_t need = phf_ozaki_dgemm_noalloc_scratch_bytes(m, n, k, slices);
    if (need > kNoAllocScratchBytes) {
        set_error(PHF_ERR_UNSUPPORTED, "phf_ozaki_dgemm_noalloc: needs " + std::to_string(need) +
                                           " bytes of scratch, the static array holds " +
                                           std::to_string(kNoAllocScratchBytes));
        return PHF_ERR_UNSUPPORTED;
    }
    unsigned char *base = nullptr;
    PHF_TRY(scratch_address(&base));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long mp = oz_pad_rows(m), np = oz_pad_cols(n);
    const size_t a_bytes = oz_slice_bytes(mp, k, slices), b_bytes = oz_slice_bytes(np, k, slices);
    signed char *As = reinterpret_cast<signed char *>(base);
    signed char *Bs = reinterpret_cast<signed char *>(base + align256(a_bytes));
    int *ea = reinterpret_cast<int *>(base + align256(a_bytes) + align256(b_bytes));
    int *eb = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(ea) + align256(mp * sizeof(int)));
    int *err = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(eb) + align256(np * sizeof(int)));
    // the padding rows of the slices and the error flag must start at zero
    PHF_CUDA(cudaMemsetAsync(As, 0, a_bytes, st));
    PHF_CUDA(cudaMemsetAsync(Bs, 0, b_bytes, st));
    PHF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    PHF_TRY(oz_slice_rows(m, k, dA, lda, slices, mp, As, ea, st));
    PHF_TRY(oz_slice_rows(n, k, dBt, ldb, slices, np, Bs, eb, st));
    PHF_TRY(oz_gemm(m, n, k, slices, As, ea, Bs, eb, dD, ldd, 0, err, st));
    int herr = 0;
    PHF_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_error(PHF_ERR_CUDA, "phf_ozaki_dgemm_noalloc: stream synchronize failed");
        return PHF_ERR_CUDA;
    }
    if (herr) {
        set_error(PHF_ERR_CUDA, "phf_ozaki_dgemm_noalloc: pipeline wait timed out");
        return PHF_ERR_CUDA;
    }
    return PHF_OK;
}
