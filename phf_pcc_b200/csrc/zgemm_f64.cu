// FP64 strided batched complex GEMM: the building block of the plain FP64 form.
//
// C[b] = alpha * A[b] * B[b] + beta * C[b] with every operand given as a strided view
// (row stride, column stride, two batch strides, optional per-batch offsets), so that
// transposes, conjugate transposes and the column-blocked layouts of the grid-point
// batches need no copies.  A may be real (real x complex products: Cholesky vectors and
// the one-electron matrix applied to complex orbitals).
//
// Tiling: BM x BN output tile per CTA of (BM / 32) (BN / 16) warps (64 x 64, 128 x 32 and 32 x 128 on
// 8 warps; 32 x 112 on 7 and 64 x 112 on 14 for products with 97..112 output columns, such as the
// per-point products with N = 100 orbitals), k-step 16, the k-tiles staged by cp.async.
// The products run on the FP64 tensor cores (mma.sync m8n8k4 .f64): each of the 8 warps owns a
// 32 x 16 block of the tile as 4 x 2 blocks of 8 x 8, and a complex product is four real MMAs
// (re re, -im im, re im, im re), two for a real A.
#include <type_traits>

#include "phf_internal.h"

namespace phf {

namespace {

constexpr int BK = 16;

template <int BM, int BN>
__host__ __device__ constexpr int zg_threads() { return (BM / 32) * (BN / 16) * 32; }
template <int BM, int BN>
__host__ __device__ constexpr int zg_min_blocks() { return zg_threads<BM, BN>() <= 256 ? 2 : 1; }

template <bool AREAL>
struct ATile {
    using T = typename std::conditional<AREAL, double, zc>::type;
};

__device__ __forceinline__ zc load_z(const View &v, long long off) {
    if (v.real) return zc{reinterpret_cast<const double *>(v.p)[off], 0.0};
    zc z = reinterpret_cast<const zc *>(v.p)[off];
    if (v.conj) z.y = -z.y;
    return z;
}

__device__ __forceinline__ double load_d(const View &v, long long off) {
    return reinterpret_cast<const double *>(v.p)[off];
}

// D (8 x 8) += A (8 x 4, row-major) B (4 x 8, column-major), FP64.  Lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2 (l%4) + {0, 1}].
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async(uint32_t dst, const void *src, int bytes_valid, int size) {
    if (size == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes_valid) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes_valid) : "memory");
}

// Shared-memory stages of the k loop (cp.async pipeline): three for the 64 x 64 and the 112-column
// tiles, two for the narrow tiles (their products are mostly k = 32, two k-tiles; two stages let two
// CTAs share an SM).
template <int BM, int BN>
__host__ __device__ constexpr int zg_stages() { return (BM == BN || BN == 112) ? 3 : 2; }

template <bool AREAL, int BM, int BN>
constexpr size_t zg_smem_bytes() {
    return (size_t)zg_stages<BM, BN>() * BK *
           ((BM + 1) * (AREAL ? sizeof(double) : sizeof(zc)) + (BN + 1) * sizeof(zc));
}

// BM x BN output tile, 256 threads = 8 warps of 32 x 16 (warp w: rows 32 (w / (BN/16)), columns
// 16 (w % (BN/16))).  64 x 64 serves general shapes; 128 x 32 the narrow per-point products
// (N <= 32 columns), 32 x 128 the N-row products bra^H Y and bra^H F X (m = N <= 32) over all
// points of a chunk.  Tiles of A and B reach shared memory by element-wise cp.async (16 bytes a
// complex element, 8 a real one; out-of-range elements are zero-filled) through zg_stages stages;
// conjugation is applied when fragments are read.  A real B (only the exchange-matrix build) is
// loaded with plain loads into the same stages.
template <bool AREAL, int BM, int BN>
__global__ void __launch_bounds__(zg_threads<BM, BN>(), zg_min_blocks<BM, BN>())
    zgemm_kernel(int m, int n, int k, int nb0, int ntn, zc alpha, View A, View B, zc beta, OutView C,
                 const long long *__restrict__ offs) {
    using TA = typename ATile<AREAL>::T;
    constexpr int WARPS_N = BN / 16;
    constexpr int NT = zg_threads<BM, BN>();
    static_assert(BM % 32 == 0 && BN % 16 == 0, "tile/warp mismatch");
    // elements loaded per thread and k-tile (the last round partial when NT does not divide the tile)
    constexpr int LA = (BM * BK + NT - 1) / NT, LB = (BN * BK + NT - 1) / NT;
    constexpr int PA = BM + 1, PB = BN + 1;                    // row pitches (elements)
    constexpr int ZG_STAGES = zg_stages<BM, BN>();
    extern __shared__ __align__(16) unsigned char zg_smem[];
    TA *As = reinterpret_cast<TA *>(zg_smem);                                      // [stage][kk][i]
    zc *Bs = reinterpret_cast<zc *>(zg_smem + (size_t)ZG_STAGES * BK * PA * sizeof(TA));  // [stage][kk][j]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp / WARPS_N) * 32, wc = (warp % WARPS_N) * 16;  // warp block within the tile
    const int fr = lane >> 2, fk = lane & 3;                            // fragment row / k of this lane
    const long long bz = blockIdx.x / ntn;
    const int tn = blockIdx.x - bz * ntn;
    const int row0 = blockIdx.y * BM, col0 = tn * BN;
    const long long b0 = bz % nb0, b1 = bz / nb0;
    long long oa = b0 * A.bs0 + b1 * A.bs1, ob = b0 * B.bs0 + b1 * B.bs1, oc = b0 * C.bs0 + b1 * C.bs1;
    if (offs) {
        oa += offs[3 * bz];
        ob += offs[3 * bz + 1];
        oc += offs[3 * bz + 2];
    }
    const bool a_mfast = (A.rs == 1);  // element order of the A tile loads
    const bool b_nfast = (B.cs == 1);
    const double sa = (!AREAL && A.conj) ? -1.0 : 1.0;  // imaginary-part signs (conjugated views)
    const double sb = B.conj ? -1.0 : 1.0;
    const uint32_t as_base = (uint32_t)__cvta_generic_to_shared(As);
    const uint32_t bs_base = (uint32_t)__cvta_generic_to_shared(Bs);
    const int nkt = (k + BK - 1) / BK;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * BK;
#pragma unroll
        for (int r = 0; r < LA; ++r) {
            const int e = tid + NT * r;
            if ((BM * BK) % NT != 0 && e >= BM * BK) break;
            int i, kk;
            if (a_mfast) { i = e % BM; kk = e / BM; }
            else { kk = e % BK; i = e / BK; }
            const int gi = row0 + i, gk = k0 + kk;
            const bool ok = gi < m && gk < k;
            const long long off = ok ? oa + (long long)gi * A.rs + (long long)gk * A.cs : 0;
            cp_async(as_base + (uint32_t)(((stage * BK + kk) * PA + i) * sizeof(TA)),
                     reinterpret_cast<const unsigned char *>(A.p) + off * (long long)sizeof(TA),
                     ok ? (int)sizeof(TA) : 0, (int)sizeof(TA));
        }
#pragma unroll
        for (int r = 0; r < LB; ++r) {
            const int e = tid + NT * r;
            if ((BN * BK) % NT != 0 && e >= BN * BK) break;
            int j, kk;
            if (b_nfast) { j = e % BN; kk = e / BN; }
            else { kk = e % BK; j = e / BK; }
            const int gj = col0 + j, gk = k0 + kk;
            const bool ok = gj < n && gk < k;
            const long long off = ok ? ob + (long long)gk * B.rs + (long long)gj * B.cs : 0;
            if (B.real) {
                Bs[(stage * BK + kk) * PB + j] = zc{ok ? reinterpret_cast<const double *>(B.p)[off] : 0.0, 0.0};
            } else {
                cp_async(bs_base + (uint32_t)(((stage * BK + kk) * PB + j) * sizeof(zc)),
                         reinterpret_cast<const zc *>(B.p) + off, ok ? 16 : 0, 16);
            }
        }
    };

    double cr[4][2][2], ci[4][2][2];  // 8 x 8 blocks (bi, bj): real and imaginary accumulators
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;

#pragma unroll
    for (int st = 0; st < ZG_STAGES - 1; ++st) {
        if (st < nkt) load_stage(st, st);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kt = 0; kt < nkt; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(ZG_STAGES - 2) : "memory");
        __syncthreads();  // stage kt landed for every thread; stage kt - 1 is no longer read
        const int stage = kt % ZG_STAGES;
        const TA *At = As + (size_t)stage * BK * PA;
        const zc *Bt = Bs + (size_t)stage * BK * PB;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            zc b[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                b[j] = Bt[(kk + fk) * PB + wc + 8 * j + fr];
                b[j].y *= sb;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                TA a = At[(kk + fk) * PA + wr + 8 * i + fr];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if constexpr (AREAL) {
                        dmma884(cr[i][j], a, b[j].x);
                        dmma884(ci[i][j], a, b[j].y);
                    } else {
                        const double ay = a.y * sa;
                        dmma884(cr[i][j], a.x, b[j].x);
                        dmma884(cr[i][j], -ay, b[j].y);
                        dmma884(ci[i][j], a.x, b[j].y);
                        dmma884(ci[i][j], ay, b[j].x);
                    }
                }
            }
        }
        const int kn = kt + ZG_STAGES - 1;  // refill the stage computed in the previous iteration
        if (kn < nkt) load_stage(kn % ZG_STAGES, kn);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = row0 + wr + 8 * i + fr;
        if (gi >= m) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = col0 + wc + 8 * j + 2 * fk + h;
                if (gj >= n) continue;
                long long off = oc + (long long)gi * C.rs + (long long)gj * C.cs;
                zc v = alpha * zc{cr[i][j][h], ci[i][j][h]};
                if (C.real) {
                    double *cp = reinterpret_cast<double *>(C.p);
                    cp[off] = use_beta ? v.x + beta.x * cp[off] : v.x;
                } else {
                    if (use_beta) v = v + beta * C.p[off];
                    C.p[off] = v;
                }
            }
    }
}

template <int BM, int BN>
int launch_tile(int m, int n, int k, int nb0, int nb1, zc alpha, const View &A, const View &B, zc beta,
                const OutView &C, const long long *offs, cudaStream_t st) {
    const int ntn = (n + BN - 1) / BN, ntm = (m + BM - 1) / BM;
    const long long nbatch = (long long)nb0 * nb1;
    const long long gx = nbatch * ntn;
    if (gx > 2147483647LL || ntm > 65535) {
        set_error(PHF_ERR_ARG, "zgemm_strided: grid too large");
        return PHF_ERR_ARG;
    }
    dim3 grid((unsigned)gx, (unsigned)ntm, 1);
    if (A.real) {
        constexpr size_t smem = zg_smem_bytes<true, BM, BN>();
        PHF_CUDA(cudaFuncSetAttribute(zgemm_kernel<true, BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        ProfScope prof(st, -1);
        zgemm_kernel<true, BM, BN><<<grid, zg_threads<BM, BN>(), smem, st>>>(m, n, k, nb0, ntn, alpha, A, B, beta, C,
                                                                             offs);
    } else {
        constexpr size_t smem = zg_smem_bytes<false, BM, BN>();
        PHF_CUDA(cudaFuncSetAttribute(zgemm_kernel<false, BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        ProfScope prof(st, -1);
        zgemm_kernel<false, BM, BN><<<grid, zg_threads<BM, BN>(), smem, st>>>(m, n, k, nb0, ntn, alpha, A, B, beta,
                                                                              C, offs);
    }
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

// Tile shape 0 = 64 x 64, 1 = 128 x 32, 2 = 32 x 128, 3 = 32 x 112, 4 = 64 x 112.
int launch_choice(int tile, int m, int n, int k, int nb0, int nb1, zc alpha, const View &A, const View &B, zc beta,
                  const OutView &C, const long long *offs, cudaStream_t st) {
    if (tile == 1) return launch_tile<128, 32>(m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
    if (tile == 2) return launch_tile<32, 128>(m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
    if (tile == 3) return launch_tile<32, 112>(m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
    if (tile == 4) return launch_tile<64, 112>(m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
    return launch_tile<64, 64>(m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
}

}  // namespace

// The tile comes from the launch tuner's table when the shape was tuned, else from rules set by
// measurements of the per-point products: 128 x 32 for at most 32 output columns and at least 96
// rows, 32 x 128 in the transposed case, 32 x 112 for 97..112 output columns (one column tile where
// 64 x 64 would pad 100 columns to 128), 64 x 64 otherwise.
int zgemm_strided(int m, int n, int k, int nb0, int nb1, zc alpha, const View &A, const View &B, zc beta,
                  const OutView &C, const long long *offs, cudaStream_t st) {
    if (m <= 0 || n <= 0 || nb0 <= 0 || nb1 <= 0) return PHF_OK;
    if (k <= 0) {
        set_error(PHF_ERR_ARG, "zgemm_strided: k <= 0");
        return PHF_ERR_ARG;
    }
    const TuneKey key{0, (long long)m, (long long)n, (long long)k, (long long)nb0 * 65536 + nb1,
                      (long long)(A.real * 4 + B.real * 2 + C.real) * 2 + (offs != nullptr)};
    if (t_tune_record)
        t_tune_record->push_back({key, {0, 1, 2, 3, 4}, [=](int tile, cudaStream_t s) {
                                      return launch_choice(tile, m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, s);
                                  }});
    int tile = tuned_choice(key);
    if (tile < 0) tile = (n <= 32 && m >= 96) ? 1 : ((m <= 32 && n >= 96) ? 2 : ((n > 96 && n <= 112) ? 3 : 0));
    return launch_choice(tile, m, n, k, nb0, nb1, alpha, A, B, beta, C, offs, st);
}

}  // namespace phf
