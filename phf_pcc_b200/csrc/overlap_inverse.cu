// Batched FP64 complex inverse, determinant and log-determinant of the rotated overlaps
// S_w = bra^H R_w ket (N x N): one warp per grid point for N <= 32, else one CTA of 32 x 32 threads
// per grid point, the matrix resident in shared memory.
//
// Replaces InvertC (ZGETRF + ZGETRI) and determinantC (ZGETRF) of PHF_fort/Wrappers.f90:195-336
// as called from RDM (PHF_fort/PHFTools.f90:259-260).  Algorithm: in-place Gauss-Jordan
// elimination with partial (row) pivoting -- the pivot is the first row of maximal |re| + |im|
// in the column, the choice LAPACK's izamax makes -- followed by the column interchanges
// in reverse order.  The pivots are those of LU with partial pivoting, so
//   det S = (-1)^{#interchanges} * prod(pivots),
//   log det S = sum log|pivot| + i (sum arg(pivot) + pi #interchanges).
// A zero pivot is reported as status 1 (the reference STOPs "Error in ZGetRF"); a
// non-finite entry as status 2.  Both are OR-ed into *flag and the outputs of that grid
// point are zeroed.
#include "phf_common.cuh"

namespace phf {

namespace {

// One CTA of 32 x 32 threads per grid point (N > 32): thread (ty, tx) updates the elements of rows
// ty + 32 m and columns tx + 32 q, so a Gauss-Jordan step is four barriers -- the pivot search is one
// warp's shuffle arg-max -- and no index division.  Element updates, pivot choice and the determinant
// are those of the algorithm above, operation for operation.
constexpr int GJ_T = 32;  // threads per row and per column of the CTA

__global__ void __launch_bounds__(GJ_T *GJ_T) gj_inverse_kernel(int N, const zc *__restrict__ S, long long s_rs,
                                                                 long long s_bs, zc *__restrict__ Sinv, long long i_rs,
                                                                 long long i_bs, zc *__restrict__ det,
                                                                 zc *__restrict__ logdet, int *__restrict__ flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    zc *A = reinterpret_cast<zc *>(smem_raw);                 // N*N, row-major
    zc *rowk = A + (size_t)N * N;                             // N
    zc *colk = rowk + N;                                      // N
    int *perm = reinterpret_cast<int *>(colk + N);            // N
    __shared__ int s_bad, s_piv;
    __shared__ double s_pv;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * GJ_T + tx;
    constexpr int NTH = GJ_T * GJ_T;
    const long long b = blockIdx.x;
    const zc *Sb = S + b * s_bs;
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int i = ty; i < N; i += GJ_T)
        for (int j = tx; j < N; j += GJ_T) {
            const zc v = Sb[(long long)i * s_rs + j];
            if (!isfinite(v.x) || !isfinite(v.y)) s_bad = 2;
            A[i * N + j] = v;
        }
    __syncthreads();

    double logabs = 0.0, phase = 0.0;  // kept by thread 0
    zc d = mkz(1.0, 0.0);
    int nswap = 0;
    for (int k = 0; k < N && s_bad == 0; ++k) {
        // pivot search (warp 0): first index of the maximal |re| + |im| in rows k..N-1 of column k
        if (ty == 0) {
            double best = -1.0;
            int bi = N;
            for (int i = k + tx; i < N; i += GJ_T) {
                const double a = abs1(A[i * N + k]);
                if (a > best) {
                    best = a;
                    bi = i;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (tx == 0) {
                s_piv = bi;
                s_pv = best;
            }
        }
        __syncthreads();
        const int p = s_piv;
        const double pv = s_pv;
        if (!(pv > 0.0)) {  // exactly singular (or NaN pivot)
            if (tid == 0) s_bad = (pv == 0.0) ? 1 : 2;
            __syncthreads();
            break;
        }
        if (p != k && tid < N) {
            const zc t = A[k * N + tid];
            A[k * N + tid] = A[p * N + tid];
            A[p * N + tid] = t;
        }
        if (tid == 0) perm[k] = p;
        __syncthreads();
        const zc piv = A[k * N + k];
        if (tid == 0) {  // running determinant and log-determinant
            d = d * piv;
            logabs += log(hypot(piv.x, piv.y));
            phase += atan2(piv.y, piv.x);
            if (p != k) {
                d = mkz(-d.x, -d.y);
                ++nswap;
            }
        }
        const zc inv = divz(mkz(1.0, 0.0), piv);
        // scaled pivot row (with 1/piv in column k) and the saved column k
        if (tid < N) rowk[tid] = (tid == k) ? inv : A[k * N + tid] * inv;
        else if (tid < 2 * N && tid - N < NTH) colk[tid - N] = A[(tid - N) * N + k];
        __syncthreads();
        for (int i = ty; i < N; i += GJ_T) {
            const zc ci = colk[i];
            for (int j = tx; j < N; j += GJ_T) {
                const int e = i * N + j;
                if (i == k) {
                    A[e] = rowk[j];
                } else {
                    const zc a = (j == k) ? mkz(0.0, 0.0) : A[e];
                    A[e] = a - ci * rowk[j];
                }
            }
        }
        __syncthreads();
    }
    const int bad = s_bad;
    if (bad == 0) {
        // undo the row interchanges as column interchanges, in reverse order
        for (int k = N - 1; k >= 0; --k) {
            const int p = perm[k];
            if (p != k && tid < N) {
                const zc t = A[tid * N + k];
                A[tid * N + k] = A[tid * N + p];
                A[tid * N + p] = t;
            }
            __syncthreads();
        }
    }
    zc *Ib = Sinv + b * i_bs;
    for (int i = ty; i < N; i += GJ_T)
        for (int j = tx; j < N; j += GJ_T) Ib[(long long)i * i_rs + j] = bad ? mkz(0.0, 0.0) : A[i * N + j];
    if (tid == 0) {
        if (bad) {
            det[b] = mkz(0.0, 0.0);
            logdet[b] = mkz(-INFINITY, 0.0);
            atomicOr(flag, bad);
        } else {
            det[b] = d;
            const double pi = 3.14159265358979323846;
            double ph = fmod(phase + pi * (nswap & 1), 2.0 * pi);
            if (ph > pi) ph -= 2.0 * pi;
            if (ph <= -pi) ph += 2.0 * pi;
            logdet[b] = mkz(logabs, ph);
        }
    }
}

// 32 < N <= 100: the matrix held in registers.  A CTA of R x C threads (R = ceil(N / MR),
// C = ceil(N / MC)) per grid point; thread (r, c) keeps the MR x MC elements of rows r + R m and
// columns c + C q for the whole elimination, so a step reads and writes no matrix element through
// shared memory: only the pivot column (N values), the scaled pivot row (N values) and one
// candidate per thread row pass through it, with two barriers per step.
//
// Rows are not interchanged.  Step k takes as pivot the eligible row p (not pivoted before) of
// maximal |re| + |im| in column k; ties go to the row that the interchanging form would hold at the
// lowest position, so the pivot sequence, the interchange count and every element update are those of
// gj_inverse_kernel (the positions are tracked in shared memory: pos[row], row_at[position]).  With
// p_k the pivot row of step k, the stored result E satisfies E[p_j][k] = inv(S)[j][p_k], which the
// write-out undoes: element (row, col) goes to inv(S)[step_of_row[row]][piv_row[col]].
constexpr int GR_NMAX = 128;  // bound of the shared pivot arrays

template <int MR, int MC, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    gj_inverse_reg_kernel(int N, int R, int C, const zc *__restrict__ S, long long s_rs, long long s_bs,
                          zc *__restrict__ Sinv, long long i_rs, long long i_bs, zc *__restrict__ det,
                          zc *__restrict__ logdet, int *__restrict__ flag) {
    // The thread grid covers rows 0 .. R MR - 1 and columns 0 .. C MC - 1; the entries outside the
    // N x N matrix are zero and stay zero (their column entries and pivot-row entries are zero in
    // every step before step N), are never taken as pivots before step N (value 0, and positions
    // above every row of the matrix), and are not written out.  So no update needs a bounds test.
    // colk alternates between two buffers by step parity: step k's column is still read in the update
    // phase after the second barrier, while the owners of column k + 1 may already publish theirs
    __shared__ zc rowk[GR_NMAX], colk2[2][GR_NMAX], pivs[GR_NMAX];
    __shared__ int pos[GR_NMAX], row_at[GR_NMAX], step_of_row[GR_NMAX], piv_row[GR_NMAX];
    __shared__ double cand_v[32];
    __shared__ int cand_pos[32], cand_row[32];
    __shared__ int s_bad;

    const int tid = threadIdx.x, lane = tid & 31;
    const bool own = tid < R * C;
    const int r = own ? tid / C : 0, c = own ? tid - (tid / C) * C : 0;
    const int nrow = R * MR;
    const long long b = blockIdx.x;
    const zc *Sb = S + b * s_bs;
    if (tid == 0) s_bad = 0;
    for (int i = tid; i < nrow; i += blockDim.x) {
        pos[i] = i;
        row_at[i] = i;
    }
    __syncthreads();
    zc a[MR][MC];
#pragma unroll
    for (int m = 0; m < MR; ++m)
#pragma unroll
        for (int q = 0; q < MC; ++q) {
            const int row = r + R * m, col = c + C * q;
            zc v = mkz(0.0, 0.0);
            if (own && row < N && col < N) {
                v = Sb[(long long)row * s_rs + col];
                if (!isfinite(v.x) || !isfinite(v.y)) s_bad = 2;
            }
            a[m][q] = v;
        }
    __syncthreads();

    int nswap = 0;  // kept by thread 0
    for (int k = 0; k < N && s_bad == 0; ++k) {
        zc *colk = colk2[k & 1];
        // (A) the owners of column k (slot q with c + C q == k: one q at most) publish it, then pick
        // their best eligible row from the published values
        bool owner = false;
#pragma unroll
        for (int q = 0; q < MC; ++q) {
            if (own && c + C * q == k) {
                owner = true;
#pragma unroll
                for (int m = 0; m < MR; ++m) colk[r + R * m] = a[m][q];
            }
        }
        if (owner) {
            double best = -1.0;
            int bpos = GR_NMAX, brow = -1;
            for (int row = r; row < nrow; row += R) {
                const int ps = pos[row];
                if (ps >= k) {
                    const double av = abs1(colk[row]);
                    if (av > best || (av == best && ps < bpos)) {
                        best = av;
                        bpos = ps;
                        brow = row;
                    }
                }
            }
            cand_v[r] = best;
            cand_pos[r] = bpos;
            cand_row[r] = brow;
        }
        __syncthreads();
        // (B) every warp reduces the R candidates: maximal value, then lowest position
        double pv = lane < R ? cand_v[lane] : -1.0;
        int pp = lane < R ? cand_pos[lane] : GR_NMAX;
        int p = lane < R ? cand_row[lane] : -1;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, pv, off);
            const int op = __shfl_xor_sync(0xffffffffu, pp, off);
            const int orow = __shfl_xor_sync(0xffffffffu, p, off);
            if (ov > pv || (ov == pv && op < pp)) {
                pv = ov;
                pp = op;
                p = orow;
            }
        }
        if (!(pv > 0.0)) {  // exactly singular (or NaN pivot): every thread leaves at the same step
            if (tid == 0) s_bad = (pv == 0.0) ? 1 : 2;
            break;
        }
        const zc piv = colk[p];
        if (own && r == p % R) {  // the owners of row p write the scaled pivot row
            const zc inv = divz(mkz(1.0, 0.0), piv);
            const int mp = p / R;
#pragma unroll
            for (int m = 0; m < MR; ++m)
                if (m == mp) {
#pragma unroll
                    for (int q = 0; q < MC; ++q) {
                        const int col = c + C * q;
                        rowk[col] = (col == k) ? inv : a[m][q] * inv;
                    }
                }
        }
        if (tid == 0) {  // pivots (det and log det are formed from them at the end) and the positions
            pivs[k] = piv;
            if (pp != k) {
                ++nswap;
                const int q = row_at[k];
                row_at[pp] = q;
                pos[q] = pp;
                row_at[k] = p;
                pos[p] = k;
            }
            step_of_row[p] = k;
            piv_row[k] = p;
        }
        __syncthreads();
        // (C) rank-1 update of the register-resident elements
        if (own) {
            zc rk[MC];
#pragma unroll
            for (int q = 0; q < MC; ++q) rk[q] = rowk[c + C * q];
#pragma unroll
            for (int m = 0; m < MR; ++m) {
                if (r + R * m == p) {
#pragma unroll
                    for (int q = 0; q < MC; ++q) a[m][q] = rk[q];
                } else {
                    const zc ci = colk[r + R * m];
#pragma unroll
                    for (int q = 0; q < MC; ++q) {
                        const zc x = (c + C * q == k) ? mkz(0.0, 0.0) : a[m][q];
                        a[m][q] = x - ci * rk[q];
                    }
                }
            }
        }
    }
    __syncthreads();
    const int bad = s_bad;
    zc *Ib = Sinv + b * i_bs;
    if (own) {
#pragma unroll
        for (int m = 0; m < MR; ++m)
#pragma unroll
            for (int q = 0; q < MC; ++q) {
                const int row = r + R * m, col = c + C * q;
                if (row < N && col < N) {
                    if (bad)
                        Ib[(long long)row * i_rs + col] = mkz(0.0, 0.0);
                    else
                        Ib[(long long)step_of_row[row] * i_rs + piv_row[col]] = a[m][q];
                }
            }
    }
    if (tid == 0) {
        if (bad) {
            det[b] = mkz(0.0, 0.0);
            logdet[b] = mkz(-INFINITY, 0.0);
            atomicOr(flag, bad);
        } else {
            // det = (-1)^{#interchanges} prod(pivots), the product and sums taken in pivot order
            zc d = mkz(1.0, 0.0);
            double logabs = 0.0, phase = 0.0;
            for (int k = 0; k < N; ++k) {
                const zc piv = pivs[k];
                d = d * piv;
                logabs += log(hypot(piv.x, piv.y));
                phase += atan2(piv.y, piv.x);
            }
            if (nswap & 1) d = mkz(-d.x, -d.y);
            det[b] = d;
            const double pi = 3.14159265358979323846;
            double ph = fmod(phase + pi * (nswap & 1), 2.0 * pi);
            if (ph > pi) ph -= 2.0 * pi;
            if (ph <= -pi) ph += 2.0 * pi;
            logdet[b] = mkz(logabs, ph);
        }
    }
}

// N <= 32: one warp per matrix (lane j owns column j), four matrices per CTA.  The same
// Gauss-Jordan steps as gj_inverse_kernel -- pivot = first index of the largest |re| + |im| in rows
// k..N-1 of column k, identical element updates -- but warp-synchronous: the pivot search is a
// shuffle arg-max and the steps are separated by __syncwarp only.  The pivots are kept and lane 0
// forms det and log det from them at the end, in pivot order.
constexpr int WI_WARPS = 4, WI_P = 33;  // matrices per CTA, row pitch (complex) of the shared copy

__host__ __device__ constexpr size_t wi_warp_bytes() { return (size_t)(32 * WI_P + 64) * sizeof(zc) + 32 * sizeof(int); }

__global__ void __launch_bounds__(WI_WARPS * 32) gj_inverse_warp_kernel(
    int N, int batch, const zc *__restrict__ S, long long s_rs, long long s_bs, zc *__restrict__ Sinv, long long i_rs,
    long long i_bs, zc *__restrict__ det, zc *__restrict__ logdet, int *__restrict__ flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long b = (long long)blockIdx.x * WI_WARPS + warp;
    if (b >= batch) return;  // the whole warp leaves; nothing below synchronises beyond the warp
    unsigned char *base = smem_raw + (size_t)warp * wi_warp_bytes();
    zc *A = reinterpret_cast<zc *>(base);  // N x N, row i at A + i WI_P
    zc *colk = A + 32 * WI_P;              // saved column k
    zc *pivs = colk + 32;                  // pivots in order
    int *perm = reinterpret_cast<int *>(pivs + 32);
    const unsigned full = 0xffffffffu;
    const bool own = lane < N;

    const zc *Sb = S + b * s_bs;
    int bad = 0;
    if (own) {
        for (int i0 = 0; i0 < N; i0 += 8) {  // eight global loads in flight, then the shared stores
            zc v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (i0 + u < N) v[u] = Sb[(long long)(i0 + u) * s_rs + lane];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (i0 + u < N) {
                    if (!isfinite(v[u].x) || !isfinite(v[u].y)) bad = 2;
                    A[(i0 + u) * WI_P + lane] = v[u];
                }
        }
    }
    bad = __reduce_max_sync(full, bad);
    __syncwarp();

    for (int k = 0; k < N && bad == 0; ++k) {
        double a = -1.0;
        int idx = N;
        if (lane >= k && lane < N) {
            const double v = abs1(A[lane * WI_P + k]);
            if (v > a) {  // NaN never becomes a candidate
                a = v;
                idx = lane;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double oa = __shfl_xor_sync(full, a, off);
            const int oi = __shfl_xor_sync(full, idx, off);
            if (oa > a || (oa == a && oi < idx)) {
                a = oa;
                idx = oi;
            }
        }
        const int p = idx;
        if (!(a > 0.0)) {  // exactly singular (or NaN pivot)
            bad = (a == 0.0) ? 1 : 2;
            break;
        }
        if (p != k && own) {
            const zc t = A[k * WI_P + lane];
            A[k * WI_P + lane] = A[p * WI_P + lane];
            A[p * WI_P + lane] = t;
        }
        __syncwarp();
        const zc piv = A[k * WI_P + k];
        const zc inv = divz(mkz(1.0, 0.0), piv);
        zc rk = mkz(0.0, 0.0);
        if (own) {
            rk = (lane == k) ? inv : A[k * WI_P + lane] * inv;
            colk[lane] = A[lane * WI_P + k];
        }
        if (lane == 0) {
            pivs[k] = piv;
            perm[k] = p;
        }
        __syncwarp();
        if (own) {  // rows in batches of eight: loads, then arithmetic, then stores (latencies overlap)
            for (int i0 = 0; i0 < N; i0 += 8) {
                zc av[8], cv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int i = i0 + u;
                    if (i < N) {
                        av[u] = A[i * WI_P + lane];
                        cv[u] = colk[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int i = i0 + u;
                    if (i < N) {
                        if (i == k) {
                            av[u] = rk;
                        } else {
                            const zc x = (lane == k) ? mkz(0.0, 0.0) : av[u];
                            av[u] = x - cv[u] * rk;
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (i0 + u < N) A[(i0 + u) * WI_P + lane] = av[u];
            }
        }
        __syncwarp();
    }
    if (bad == 0) {
        // undo the row interchanges as column interchanges, in reverse order (lane i swaps row i)
        for (int k = N - 1; k >= 0; --k) {
            const int p = perm[k];
            if (p != k && own) {
                const zc t = A[lane * WI_P + k];
                A[lane * WI_P + k] = A[lane * WI_P + p];
                A[lane * WI_P + p] = t;
            }
            __syncwarp();
        }
    }
    zc *Ib = Sinv + b * i_bs;
    for (int i = 0; i < N; ++i)
        if (own) Ib[(long long)i * i_rs + lane] = bad ? mkz(0.0, 0.0) : A[i * WI_P + lane];
    if (lane == 0) {
        if (bad) {
            det[b] = mkz(0.0, 0.0);
            logdet[b] = mkz(-INFINITY, 0.0);
            atomicOr(flag, bad);
        } else {
            zc d = mkz(1.0, 0.0);
            double logabs = 0.0, phase = 0.0;
            int nswap = 0;
            for (int k = 0; k < N; ++k) {
                const zc piv = pivs[k];
                d = d * piv;
                logabs += log(hypot(piv.x, piv.y));
                phase += atan2(piv.y, piv.x);
                if (perm[k] != k) {
                    d = mkz(-d.x, -d.y);
                    ++nswap;
                }
            }
            det[b] = d;
            const double pi = 3.14159265358979323846;
            double ph = fmod(phase + pi * (nswap & 1), 2.0 * pi);
            if (ph > pi) ph -= 2.0 * pi;
            if (ph <= -pi) ph += 2.0 * pi;
            logdet[b] = mkz(logabs, ph);
        }
    }
}

}  // namespace

size_t overlap_inverse_smem(int N) { return (size_t)N * N * sizeof(zc) + 2 * (size_t)N * sizeof(zc) + N * sizeof(int); }

int overlap_inverse(int N, int batch, const zc *S, long long s_rs, long long s_bs, zc *Sinv, long long i_rs,
                    long long i_bs, zc *det, zc *logdet, int *flag, cudaStream_t st) {
    if (N <= 32) {
        const size_t smem = WI_WARPS * wi_warp_bytes();
        PHF_CUDA(cudaFuncSetAttribute(gj_inverse_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ProfScope prof(st, PROF_INVERSE);
        gj_inverse_warp_kernel<<<(unsigned)((batch + WI_WARPS - 1) / WI_WARPS), WI_WARPS * 32, smem, st>>>(
            N, batch, S, s_rs, s_bs, Sinv, i_rs, i_bs, det, logdet, flag);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    if (N <= 100) {
        // register-resident elimination: MR x MC elements per thread, R x C <= 512 threads, R <= 32
        const bool small = N <= 64;
        const int MR = small ? 4 : 5, MC = 4;
        const int R = (N + MR - 1) / MR, C = (N + MC - 1) / MC;
        const unsigned threads = (unsigned)((R * C + 31) / 32 * 32);
        ProfScope prof(st, PROF_INVERSE);
        if (small)
            gj_inverse_reg_kernel<4, 4, 256, 2><<<batch, threads, 0, st>>>(N, R, C, S, s_rs, s_bs, Sinv, i_rs, i_bs,
                                                                            det, logdet, flag);
        else
            gj_inverse_reg_kernel<5, 4, 512, 1><<<batch, threads, 0, st>>>(N, R, C, S, s_rs, s_bs, Sinv, i_rs, i_bs,
                                                                            det, logdet, flag);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    size_t smem = overlap_inverse_smem(N);
    PHF_CUDA(cudaFuncSetAttribute(gj_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ProfScope prof(st, PROF_INVERSE);
    gj_inverse_kernel<<<batch, dim3(GJ_T, GJ_T), smem, st>>>(N, S, s_rs, s_bs, Sinv, i_rs, i_bs, det, logdet, flag);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

}  // namespace phf

extern "C" int phf_overlap_inverse(int n, int batch, const double *dS, double *dSinv, double *ddet, double *dlogdet,
                                   int *dflag, void *stream) {
    using namespace phf;
    set_error(PHF_OK, "");
    if (n <= 0 || batch <= 0 || !dS || !dSinv || !ddet || !dlogdet || !dflag) {
        set_error(PHF_ERR_ARG, "phf_overlap_inverse: bad sizes or null pointer");
        return PHF_ERR_ARG;
    }
    if (n > 112) {  // the shared-memory form holds n^2 complex per CTA
        set_error(PHF_ERR_UNSUPPORTED, "phf_overlap_inverse: n above the inverse's limit of 112");
        return PHF_ERR_UNSUPPORTED;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long nn = (long long)n * n;
    PHF_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), st));
    PHF_TRY(overlap_inverse(n, batch, reinterpret_cast<const zc *>(dS), n, nn, reinterpret_cast<zc *>(dSinv), n, nn,
                            reinterpret_cast<zc *>(ddet), reinterpret_cast<zc *>(dlogdet), dflag, st));
    int flag = 0;
    PHF_CUDA(cudaMemcpyAsync(&flag, dflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        set_error(PHF_ERR_CUDA, "stream synchronize failed");
        return PHF_ERR_CUDA;
    }
    if (flag & 1) {
        set_error(PHF_ERR_SINGULAR, "phf_overlap_inverse: an exactly singular matrix");
        return PHF_ERR_SINGULAR;
    }
    if (flag & 2) {
        set_error(PHF_ERR_NONFINITE, "phf_overlap_inverse: a non-finite entry");
        return PHF_ERR_NONFINITE;
    }
    return PHF_OK;
}
