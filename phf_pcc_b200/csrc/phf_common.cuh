// Shared definitions for the B200 projected-HF grid kernel library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/phf_b200.h"

namespace phf {

// ---------------------------------------------------------------- complex helpers
struct __align__(16) zc {
    double x, y;
};

__host__ __device__ __forceinline__ zc mkz(double r, double i = 0.0) { return zc{r, i}; }
__host__ __device__ __forceinline__ zc operator+(zc a, zc b) { return zc{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ zc operator-(zc a, zc b) { return zc{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ zc operator*(zc a, zc b) {
    return zc{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ zc operator*(double s, zc a) { return zc{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ zc conjz(zc a) { return zc{a.x, -a.y}; }
__host__ __device__ __forceinline__ double abs1(zc a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ zc divz(zc a, zc b) {
    // Smith's algorithm for complex division
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return zc{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
    } else {
        double r = b.x / b.y, den = b.x * r + b.y;
        return zc{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
    }
}

// ---------------------------------------------------------------- errors
struct Error {
    int status;
    std::string msg;
};

void set_error(int status, const std::string &msg);
int last_status();

#define PHF_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            ::phf::set_error(PHF_ERR_CUDA, std::string(#call " -> ") + cudaGetErrorString(e_)); \
            return PHF_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

#define PHF_CHECK_LAUNCH()                                                                     \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess) {                                                               \
            ::phf::set_error(PHF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
            return PHF_ERR_CUDA;                                                               \
        }                                                                                      \
    } while (0)

#define PHF_TRY(expr)                   \
    do {                                \
        int s_ = (expr);                \
        if (s_ != PHF_OK) return s_;    \
    } while (0)

// ---------------------------------------------------------------- strided matrix views
// Element (i, j) of batch (b0, b1) lives at p + i*rs + j*cs + b0*bs0 + b1*bs1 (+ off[b] when an
// offset table is given).  Complex views count in zc elements, real views in doubles.
struct View {
    const void *p = nullptr;
    long long rs = 0, cs = 0, bs0 = 0, bs1 = 0;
    int conj = 0;  // conjugate complex elements on load
    int real = 0;  // elements are real doubles
};

struct OutView {
    zc *p = nullptr;  // complex output, or double output when real != 0
    long long rs = 0, cs = 0, bs0 = 0, bs1 = 0;
    int real = 0;     // store only the real part into a double array
};

// Launch counter: every kernel this library launches increments it (host side).
extern unsigned long long g_launches;

// Optional per-kernel-class timing with CUDA events recorded on the launching stream
// (phf_profile_enable / phf_profile_read).  Classes:
enum ProfClass { PROF_JK = 0, PROF_GEMM = 1, PROF_INVERSE = 2, PROF_MEMORY = 3, PROF_NCLASS = 4 };
void prof_set_class(int cls);  // class of the launches that follow (thread-local)
int prof_class();
struct ProfScope {             // records a start event now and an end event at scope exit
    cudaStream_t st;
    int slot;
    ProfScope(cudaStream_t s, int cls);
    ~ProfScope();
};

// C[b] = alpha * A[b] * B[b] + beta * C[b]  (FP64 complex, or real x complex when A.real)
// Batches: b = b1 * nb0 + b0.  When offs != nullptr it holds 3 * nbatch long long element
// offsets (a, b, c) per batch that are added on top of the strides.
int zgemm_strided(int m, int n, int k, int nb0, int nb1, zc alpha, const View &A, const View &B, zc beta,
                  const OutView &C, const long long *offs, cudaStream_t st);

}  // namespace phf
