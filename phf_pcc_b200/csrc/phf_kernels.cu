// Memory-bound kernels of the projected-HF pipeline: traces of the Cholesky-projected
// overlaps, the energy/gradient epilogue, the weighted (Wigner x point-group) accumulation
// over grid points, and layout transforms.  All reductions run in a fixed order, so two
// runs give bit-identical results.
#include "phf_common.cuh"

namespace phf {

namespace {

constexpr int NT = 256;

// block-wide complex sum with a fixed tree (deterministic for a fixed block size)
__device__ zc block_sum(zc v, zc *sh) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s) sh[tid] = sh[tid] + sh[tid + s];
        __syncthreads();
    }
    zc r = sh[0];
    __syncthreads();
    return r;
}

// For each Cholesky vector L and grid point w, with T_Lw = bra^H B_L X_w (N x N):
//   d = tr T, e2part[w*L_tot + L] = d^2 - tr(T T), and T <- d I - T  (in place).
// T_Lw is the block at rows L*N, columns w*N of a (L_tot*N) x ldT matrix.
__global__ void __launch_bounds__(NT) tprime_kernel(int Ltot, int N, zc *T, long long ldT, zc *e2part) {
    __shared__ zc sh[NT];
    const long long L = blockIdx.x, w = blockIdx.y;
    zc *base = T + L * N * ldT + w * N;
    zc dd = mkz(0, 0), t2 = mkz(0, 0);
    for (int j = threadIdx.x; j < N; j += NT) dd = dd + base[(long long)j * ldT + j];
    for (int e = threadIdx.x; e < N * N; e += NT) {
        int j = e / N, jp = e - j * N;
        t2 = t2 + base[(long long)j * ldT + jp] * base[(long long)jp * ldT + j];
    }
    dd = block_sum(dd, sh);
    t2 = block_sum(t2, sh);
    if (threadIdx.x == 0) e2part[w * Ltot + L] = dd * dd - t2;
    for (int e = threadIdx.x; e < N * N; e += NT) {
        int j = e / N, jp = e - j * N;
        long long o = (long long)j * ldT + jp;
        zc t = base[o];
        base[o] = (j == jp) ? (dd - t) : mkz(-t.x, -t.y);
    }
}

// out[r] = scale * sum_c in[r * ncols + c]
__global__ void __launch_bounds__(NT) rowsum_kernel(int ncols, const zc *in, zc *out, double scale) {
    __shared__ zc sh[NT];
    const long long r = blockIdx.x;
    zc s = mkz(0, 0);
    for (int c = threadIdx.x; c < ncols; c += NT) s = s + in[r * ncols + c];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[r] = scale * s;
}

// out[w] = scale * sum_{r,j} conj(C[r*N + j]) * X[r*ldX + w*N + j]   (tr(C^H X_w)), minus
// sub_scale * sub[w] when `sub` is given
__global__ void __launch_bounds__(NT) trace_conj_kernel(int M, int N, const zc *C, zc *X, long long ldX, zc *out,
                                                        double scale, const zc *add, const zc *sub, double sub_scale) {
    __shared__ zc sh[NT];
    const long long w = blockIdx.x;
    zc s = mkz(0, 0);
    for (int e = threadIdx.x; e < M * N; e += NT) {
        int r = e / N, j = e - r * N;
        const long long o = (long long)r * ldX + w * N + j;
        const zc x = X[o];
        s = s + conjz(C[e]) * x;
        if (add) X[o] = x + add[o];  // X <- X + add once the trace has read X
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[w] = sub ? scale * s - sub_scale * sub[w] : scale * s;
}

// Energy/gradient epilogue over a chunk of b grid points (Gradient, PHFTools.f90:291-308, in
// the rank-N form): with h_w = e1_w + e2_w and N_w = det S_w,
//   G <- N_w (G + h_w X)          where G already holds HX + GammaX - X W_w
//   X <- N_w X
//   scal[2w] = N_w h_w, scal[2w+1] = N_w
__global__ void __launch_bounds__(NT) epilogue_kernel(int M, int N, int b, zc *G, zc *X, long long ldX,
                                                      const zc *det, const zc *e1, const zc *e2, zc *scal) {
    const long long total = (long long)M * b * N;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        long long r = e / ((long long)b * N);
        long long c = e - r * ((long long)b * N);
        int w = (int)(c / N);
        long long o = r * ldX + c;
        zc h = e1[w] + e2[w];
        zc nd = det[w];
        zc x = X[o];
        G[o] = nd * (G[o] + h * x);
        X[o] = nd * x;
    }
    if (blockIdx.x == 0) {
        for (int w = threadIdx.x; w < b; w += NT) {
            zc h = e1[w] + e2[w];
            scal[2 * w] = det[w] * h;
            scal[2 * w + 1] = det[w];
        }
    }
}

// Neumaier compensated add of a complex term into (s, c)
__device__ __forceinline__ void neumaier(double &s, double &c, double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// Weighted accumulation over a chunk of grid points (PHFTools.f90:137-166):
//   accG[a] += sum_w Wt[s, w0 + w] * G_w,  accR[a] += sum_w Wt[s, w0 + w] * R_w,
//   accHS[a] += sum_w Wt[s, w0 + w] * (N h, N)_w      with a = slotmap[s].
// Two stages with a fixed partition, so the result does not depend on scheduling:
//   stage 1: thread (element, group q) sums the points [q*ACC_GROUP, (q+1)*ACC_GROUP) in order
//            with Neumaier compensation into part[q] (sum, compensation);
//   stage 2: thread (element) adds part[0..ngroups) in order into the running (acc, comp).
constexpr int ACC_GROUP = 32;

struct AccPart {
    double gs_r, gs_i, gc_r, gc_i, rs_r, rs_i, rc_r, rc_i;
};

__global__ void __launch_bounds__(NT) accumulate_partial_kernel(int nslot, int M, int N, int b, const zc *Wt,
                                                                long long nomega, long long w0, const zc *G,
                                                                const zc *R, long long ldX, const zc *scal,
                                                                int ngroups, AccPart *part, AccPart *part_hs,
                                                                int conj_w) {
    const long long MN = (long long)M * N;
    const long long nel = (long long)nslot * MN;
    const long long total = nel * ngroups;
    for (long long t = blockIdx.x * (long long)NT + threadIdx.x; t < total; t += (long long)gridDim.x * NT) {
        const int q = (int)(t / nel);
        const long long e = t - (long long)q * nel;
        const int s = (int)(e / MN);
        const long long rj = e - (long long)s * MN;
        const long long r = rj / N, j = rj - r * N;
        const int wa = q * ACC_GROUP, wb = min(b, wa + ACC_GROUP);
        const zc *wrow = Wt + (long long)s * nomega + w0;
        AccPart P = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int w = wa; w < wb; ++w) {
            const zc wt = conj_w ? conjz(wrow[w]) : wrow[w];
            const long long o = r * ldX + (long long)w * N + j;
            const zc tg = wt * G[o], tr = wt * R[o];
            neumaier(P.gs_r, P.gc_r, tg.x);
            neumaier(P.gs_i, P.gc_i, tg.y);
            neumaier(P.rs_r, P.rc_r, tr.x);
            neumaier(P.rs_i, P.rc_i, tr.y);
        }
        part[t] = P;
        if (rj == 0 && scal) {  // the two scalars of the slot ride on the element (s, 0, 0)
            AccPart Q = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int w = wa; w < wb; ++w) {
                const zc wt = conj_w ? conjz(wrow[w]) : wrow[w];
                const zc th = wt * scal[2 * w], ts = wt * scal[2 * w + 1];
                neumaier(Q.gs_r, Q.gc_r, th.x);
                neumaier(Q.gs_i, Q.gc_i, th.y);
                neumaier(Q.rs_r, Q.rc_r, ts.x);
                neumaier(Q.rs_i, Q.rc_i, ts.y);
            }
            part_hs[(long long)q * nslot + s] = Q;
        }
    }
}

__device__ __forceinline__ void add_part(double &s, double &c, double ps, double pc) {
    neumaier(s, c, ps);
    c += pc;
}

__global__ void __launch_bounds__(NT) accumulate_final_kernel(int nslot, int M, int N, const int *slotmap,
                                                              int ngroups, const AccPart *part,
                                                              const AccPart *part_hs, zc *accG, zc *compG, zc *accR,
                                                              zc *compR, zc *accHS, zc *compHS) {
    const long long MN = (long long)M * N;
    const long long nel = (long long)nslot * MN;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < nel; e += (long long)gridDim.x * NT) {
        const int s = (int)(e / MN);
        const long long rj = e - (long long)s * MN;
        const long long a = (long long)slotmap[s] * MN + rj;
        double gs_r = accG[a].x, gs_i = accG[a].y, gc_r = compG[a].x, gc_i = compG[a].y;
        double rs_r = accR[a].x, rs_i = accR[a].y, rc_r = compR[a].x, rc_i = compR[a].y;
        for (int q = 0; q < ngroups; ++q) {
            const AccPart P = part[(long long)q * nel + e];
            add_part(gs_r, gc_r, P.gs_r, P.gc_r);
            add_part(gs_i, gc_i, P.gs_i, P.gc_i);
            add_part(rs_r, rc_r, P.rs_r, P.rc_r);
            add_part(rs_i, rc_i, P.rs_i, P.rc_i);
        }
        accG[a] = mkz(gs_r, gs_i);
        compG[a] = mkz(gc_r, gc_i);
        accR[a] = mkz(rs_r, rs_i);
        compR[a] = mkz(rc_r, rc_i);
        if (rj == 0 && accHS) {
            const long long ah = 2LL * slotmap[s];
            double hs_r = accHS[ah].x, hs_i = accHS[ah].y, hc_r = compHS[ah].x, hc_i = compHS[ah].y;
            double ss_r = accHS[ah + 1].x, ss_i = accHS[ah + 1].y, sc_r = compHS[ah + 1].x, sc_i = compHS[ah + 1].y;
            for (int q = 0; q < ngroups; ++q) {
                const AccPart Q = part_hs[(long long)q * nslot + s];
                add_part(hs_r, hc_r, Q.gs_r, Q.gc_r);
                add_part(hs_i, hc_i, Q.gs_i, Q.gc_i);
                add_part(ss_r, sc_r, Q.rs_r, Q.rc_r);
                add_part(ss_i, sc_i, Q.rs_i, Q.rc_i);
            }
            accHS[ah] = mkz(hs_r, hs_i);
            compHS[ah] = mkz(hc_r, hc_i);
            accHS[ah + 1] = mkz(ss_r, ss_i);
            compHS[ah + 1] = mkz(sc_r, sc_i);
        }
    }
}

// a[i] += c[i]  (fold the compensation terms into the sums)
__global__ void fold_comp_kernel(long long n, zc *a, const zc *c) {
    for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT)
        a[i] = a[i] + c[i];
}

// H2r[(i M + k) M^2 + (l M + j)] = H2(i, j, k, l) with H2 in Fortran order (MakeGamma operand
// reshaped to an M^2 x M^2 matrix acting on vec(rho) with rho(l, j) at l M + j)
__global__ void permute_h2_kernel(int M, const zc *H2, zc *H2r) {
    const long long M2 = (long long)M * M, tot = M2 * M2;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long row = e / M2, col = e - row * M2;
        long long i = row / M, k = row - i * M, l = col / M, j = col - l * M;
        H2r[e] = H2[i + M * (j + M * (k + M * l))];
    }
}

// out[r*N + j] = in[rowmap[r]*ldin + j]  (row permutation of an M x N matrix, batched by blockIdx.y)
__global__ void permute_rows_kernel(int M, int N, const int *rowmap, const zc *in, long long ldin, long long bs_in,
                                    zc *out, long long bs_out) {
    const long long tot = (long long)M * N;
    const zc *src = in + blockIdx.y * bs_in;
    zc *dst = out + blockIdx.y * bs_out;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long r = e / N, j = e - r * N;
        dst[e] = src[(long long)rowmap[r] * ldin + j];
    }
}

// P[(p n + q) ldp + w] = rho_w[2p][2q] + rho_w[2p+1][2q+1]  (spin-summed density for J)
__global__ void gather_p_kernel(int n, int b, const zc *rho, zc *P, long long ldp) {
    const int M = 2 * n;
    const long long tot = (long long)n * n * b;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long pq = e / b, w = e - pq * b;
        int p = (int)(pq / n), q = (int)(pq - (long long)p * n);
        const zc *R = rho + w * (long long)M * M;
        P[pq * ldp + w] = R[(long long)(2 * p) * M + 2 * q] + R[(long long)(2 * p + 1) * M + 2 * q + 1];
    }
}

// Kin[(l n + j) ldk + 4 w + 2 sigma + tau] = rho_w[2l + sigma][2j + tau]  (exchange operand)
__global__ void gather_kin_kernel(int n, int b, const zc *rho, zc *Kin, long long ldk) {
    const int M = 2 * n;
    const long long tot = (long long)n * n * b * 4;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long lj = e / (4LL * b), c = e - lj * 4LL * b;
        long long w = c >> 2;
        int sg = (int)((c >> 1) & 1), tu = (int)(c & 1);
        int l = (int)(lj / n), j = (int)(lj - (long long)l * n);
        Kin[lj * ldk + c] = rho[w * (long long)M * M + (long long)(2 * l + sg) * M + 2 * j + tu];
    }
}

// Gamma_w[2i + sigma][2k + tau] = delta_{sigma tau} J[(i, k), w] - K_{sigma tau}[(i, k), w]
// J: complex J[(i n + k) ldj + w], or real/imaginary pairs with element (ik, c) of Jr at
//    Jr[ik jrs + c jcs], c = 2 w + part;
// K: complex Kc[(i n + k) ldk + 4 w + st], or pairs with element (ik, c) of Kr at Kr[ik krs + c kcs],
//    c = 2 (4 w + st) + part.  ksym (complex Kc only): K from its symmetric-form parts, KS of the pair
//    (min(i, k), max(i, k)) at row pair_le and KA at row n(n + 1)/2 + pair_lt (row order of the pairs),
//    K[i][k] = KS + KA for i < k, KS - KA for i > k, KS for i = k.
__global__ void assemble_gamma_kernel(int n, int b, const zc *J, long long ldj, const double *Jr, long long jrs,
                                      long long jcs, const zc *Kc, long long ldk, const double *Kr, long long krs,
                                      long long kcs, zc *Gam, int ksym, const double *h) {
    const int M = 2 * n;
    const long long tot = (long long)M * M * b;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long w = e / ((long long)M * M), rc = e - w * (long long)M * M;
        int r = (int)(rc / M), c = (int)(rc - (long long)r * M);
        int i = r >> 1, sg = r & 1, k = c >> 1, tu = c & 1;
        long long ik = (long long)i * n + k;
        int st = sg * 2 + tu;
        zc kv;
        if (Kc && ksym) {
            const long long lo = i < k ? i : k, hi = i < k ? k : i, nn = n;
            const long long ts = lo * nn - lo * (lo - 1) / 2 + (hi - lo);
            kv = Kc[ts * ldk + 4 * w + st];
            if (lo != hi) {
                const long long ta = nn * (nn + 1) / 2 + lo * (nn - 1) - lo * (lo - 1) / 2 + (hi - lo - 1);
                const zc ka = Kc[ta * ldk + 4 * w + st];
                kv = i < k ? kv + ka : kv - ka;
            }
        } else if (Kc) {
            kv = Kc[ik * ldk + 4 * w + st];
        } else {
            const long long cc = 2 * (4 * w + st);
            kv = mkz(Kr[ik * krs + cc * kcs], Kr[ik * krs + (cc + 1) * kcs]);
        }
        zc g = mkz(-kv.x, -kv.y);
        if (sg == tu) {
            if (J) g = g + J[ik * ldj + w];
            else g = g + mkz(Jr[ik * jrs + 2 * w * jcs], Jr[ik * jrs + (2 * w + 1) * jcs]);
            if (h) g.x += h[ik];
        }
        Gam[e] = g;
    }
}

// ket-side gradient: V_w += H1 C + conj(h_w) C   (V already holds Gamma_w^H C - C W_w^H; Hb = H1 C is
// null when Gamma holds H1 + J - K, whose adjoint already brought H1 C in)
__global__ void ket_prep_kernel(int M, int N, int b, const zc *Hb, const zc *bra, const zc *e1, const zc *e2, zc *V,
                                long long ld) {
    const long long total = (long long)M * b * N;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        long long r = e / ((long long)b * N), c = e - r * ((long long)b * N);
        int w = (int)(c / N), j = (int)(c - (long long)w * N);
        zc h = conjz(e1[w] + e2[w]);
        const zc hb = Hb ? Hb[r * N + j] : mkz(0.0, 0.0);
        V[r * ld + c] = V[r * ld + c] + hb + h * bra[r * N + j];
    }
}

// P_w <- conj(det_w) P_w
__global__ void scale_conj_det_kernel(int M, int N, int b, const zc *det, zc *P, long long ld) {
    const long long total = (long long)M * b * N;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        long long r = e / ((long long)b * N), c = e - r * ((long long)b * N);
        int w = (int)(c / N);
        P[r * ld + c] = conjz(det[w]) * P[r * ld + c];
    }
}

// out = (a + b) / 2
__global__ void average_kernel(long long n, const zc *a, const zc *b, zc *out) {
    for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT)
        out[i] = 0.5 * (a[i] + b[i]);
}

// Y_w = R1[il] T2[:, rem] for a spin rotation R1 that is block diagonal with one 2 x 2 block per
// spatial orbital in the interleaved order r = 2p + sigma (R1b[(il n + p) 4 + 2 sigma + tau] =
// R1[il][2p + sigma][2p + tau]): row r of Y takes two rows of T2.  Point w = w0 + wl of the chunk
// belongs to Lebedev point il = w / blk and takes column block rem = w % blk of T2; Y is row-major
// M x (bc N) with leading dimension ld, as the GEMM form writes it.
__global__ void spin_block_y_kernel(int n, int N, int bc, int w0, int blk, const zc *__restrict__ R1b,
                                    const zc *__restrict__ T2, long long ld2, zc *__restrict__ Ys, long long ld) {
    const long long cols = (long long)bc * N, total = 2LL * n * cols;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        const int r = (int)(e / cols);
        const long long c = e - (long long)r * cols;
        const int wl = (int)(c / N), j = (int)(c - (long long)wl * N);
        const int w = w0 + wl, il = w / blk, rem = w - il * blk;
        const int pp = r >> 1, sg = r & 1;
        const zc *B = R1b + ((long long)il * n + pp) * 4 + 2 * sg;
        const long long tc = (long long)rem * N + j;
        Ys[(long long)r * ld + c] = B[0] * T2[(long long)(2 * pp) * ld2 + tc] + B[1] * T2[(long long)(2 * pp + 1) * ld2 + tc];
    }
}

// Coulomb term of the tensor-core path: Gamma_w[2i + s][2k + s] += J_w(i, k) (+ h[i][k] with `h`: the
// one-electron matrix folded in, Gamma becoming the Fock matrix H1 + J - K) for both spins s, with
// J_w's real and imaginary parts at Jr[ik jrs + (2w) jcs] and Jr[ik jrs + (2w + 1) jcs] (Gamma already
// holds -K from the exchange GEMM).
__global__ void add_coulomb_diag_kernel(int n, int b, const double *Jr, long long jrs, long long jcs, zc *Gam,
                                        const double *h) {
    const int M = 2 * n;
    const long long nn = (long long)n * n, tot = 2LL * nn * b;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        const long long w = e / (2 * nn), rem = e - w * 2 * nn;
        const int sg = (int)(rem / nn);
        const long long ik = rem - (long long)sg * nn;
        const int i = (int)(ik / n), k = (int)(ik - (long long)i * n);
        zc *g = Gam + (w * M + 2 * i + sg) * M + 2 * k + sg;
        zc jv = mkz(Jr[ik * jrs + 2 * w * jcs], Jr[ik * jrs + (2 * w + 1) * jcs]);
        if (h) jv.x += h[ik];
        *g = *g + jv;
    }
}

// Symmetric and antisymmetric FP64 exchange rows of one panel from its Gram block (the symmetric
// exchange form; the tensor-core slicer slice_ek_sym_panel_kernel does the same with slices):
// pair (i, k) = pairs[t0 + r] of symmetric row r, B[l][j] = G[(i - i0) n + l][(k - k0) n + j];
// EKs[r][pair_le(l, j)] = B[l][j] + B[j][l] (l < j), B[l][l] (l = j); for i < k
// EKa[r - (i - i0) - 1][pair_lt(l, j)] = B[l][j] - B[j][l] (l < j).  Row lengths n(n+1)/2, n(n-1)/2.
// 32 x 32 tile pairs through shared memory, so that both B[l][j] and B[j][l] are read in rows.
__global__ void __launch_bounds__(256) ek_sym_panel_kernel(int n, int i0, int k0, const int *__restrict__ pairs,
                                                           long long t0, const double *__restrict__ G, long long ldg,
                                                           double *__restrict__ EKs, double *__restrict__ EKa) {
    __shared__ double T1[32 * 33], T2[32 * 33];
    const long long r = blockIdx.x, nn = n;
    const int pr = __ldg(pairs + t0 + r), i = pr >> 16, k = pr & 0xffff;
    const bool anti = i < k;
    const long long ra = r - (i - i0) - 1;
    const double *g = G + (long long)(i - i0) * n * ldg + (long long)(k - k0) * n;
    double *es = EKs + r * (nn * (nn + 1) / 2), *ea = anti ? EKa + ra * (nn * (nn - 1) / 2) : nullptr;
    const int nt = (n + 31) / 32, lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int lt = 0; lt < nt; ++lt) {
        for (int jt = lt; jt < nt; ++jt) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int a = ty + 8 * q;
                const int l1 = lt * 32 + a, j1 = jt * 32 + lane;
                T1[a * 33 + lane] = (l1 < n && j1 < n) ? g[(long long)l1 * ldg + j1] : 0.0;
                if (jt != lt) {
                    const int l2 = jt * 32 + a, j2 = lt * 32 + lane;
                    T2[a * 33 + lane] = (l2 < n && j2 < n) ? g[(long long)l2 * ldg + j2] : 0.0;
                }
            }
            __syncthreads();
            const double *U = (jt == lt) ? T1 : T2;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int a = ty + 8 * q, l = lt * 32 + a, j = jt * 32 + lane;
                if (l <= j && j < n) {
                    const double x = T1[a * 33 + lane], y = U[lane * 33 + a];
                    es[(long long)l * nn - (long long)l * (l - 1) / 2 + (j - l)] = (l == j) ? x : x + y;
                    if (anti && l < j) ea[(long long)l * (nn - 1) - (long long)l * (l - 1) / 2 + (j - l - 1)] = x - y;
                }
            }
            __syncthreads();
        }
    }
}

// Kin in the symmetric exchange form: rows t = pair_le(l, j) (pairs[t] = l << 16 | j) hold
// rho_s^{st}[l][j] = (rho_w[2l + s][2j + t] + rho_w[2j + s][2l + t]) / 2 at column 4w + st (row stride ldk);
// rows n(n+1)/2 + pair_lt(l, j), l < j, the antisymmetric halves (difference / 2).  rho_w dense M x M.
__global__ void gather_kin_sym_kernel(int n, int b, const int *__restrict__ pairs, const zc *rho, zc *Kin,
                                      long long ldk) {
    const int M = 2 * n;
    const long long nn = n, kks = nn * (nn + 1) / 2, tot = kks * b * 4;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        const long long t = e / (4LL * b), c = e - t * 4LL * b, w = c >> 2;
        const int sg = (int)((c >> 1) & 1), tu = (int)(c & 1);
        const int pr = pairs[t], l = pr >> 16, j = pr & 0xffff;
        const zc *R = rho + w * (long long)M * M;
        const zc v = R[(long long)(2 * l + sg) * M + 2 * j + tu];
        if (l == j) {
            Kin[t * ldk + c] = v;
        } else {
            const zc u = R[(long long)(2 * j + sg) * M + 2 * l + tu];
            Kin[t * ldk + c] = mkz(0.5 * (v.x + u.x), 0.5 * (v.y + u.y));
            const long long ta = kks + (long long)l * (nn - 1) - (long long)l * (l - 1) / 2 + (j - l - 1);
            Kin[ta * ldk + c] = mkz(0.5 * (v.x - u.x), 0.5 * (v.y - u.y));
        }
    }
}

// One panel of the FP64 exchange matrix from its Gram block (streamed form): for r = (i - i0) n + k,
// EKp[r][l n + j] = G[(i - i0) n + l][k n + j] (ldg, lde: row strides), i.e. (il|kj) for the panel's i.
// One CTA per output row; for fixed l the n values j are contiguous on both sides.
__global__ void ek_panel_kernel(int n, const double *__restrict__ G, long long ldg, double *__restrict__ EKp,
                                long long lde) {
    const long long r = blockIdx.x;
    const int il = (int)(r / n), k = (int)(r - (long long)il * n);
    const double *g = G + (long long)il * n * ldg + (long long)k * n;
    double *e = EKp + r * lde;
    const int kk = n * n;
    for (int t = threadIdx.x; t < kk; t += NT) {
        const int l = t / n, j = t - l * n;
        e[t] = g[(long long)l * ldg + j];
    }
}

inline int grid_for(long long n) {
    long long g = (n + NT - 1) / NT;
    if (g > 148LL * 16) g = 148LL * 16;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

int launch_tprime(int Ltot, int N, int b, zc *T, long long ldT, zc *e2part, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    tprime_kernel<<<dim3(Ltot, b), NT, 0, st>>>(Ltot, N, T, ldT, e2part);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_rowsum(int nrows, int ncols, const zc *in, zc *out, double scale, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    rowsum_kernel<<<nrows, NT, 0, st>>>(ncols, in, out, scale);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_trace_conj(int M, int N, int b, const zc *C, zc *X, long long ldX, zc *out, double scale, cudaStream_t st,
                      const zc *add, const zc *sub, double sub_scale) {
    ProfScope prof(st, PROF_MEMORY);
    trace_conj_kernel<<<b, NT, 0, st>>>(M, N, C, X, ldX, out, scale, add, sub, sub_scale);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

// G <- G + A over a chunk (M rows x b N columns, row stride ldX)
__global__ void __launch_bounds__(NT) add_inplace_kernel(long long rows, long long cols, const zc *A, zc *G,
                                                         long long ldX) {
    const long long total = rows * cols;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        const long long r = e / cols, c = e - r * cols, o = r * ldX + c;
        G[o] = G[o] + A[o];
    }
}

int launch_add_inplace(int M, int N, int b, const zc *A, zc *G, long long ldX, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    add_inplace_kernel<<<grid_for((long long)M * b * N), NT, 0, st>>>(M, (long long)b * N, A, G, ldX);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_epilogue(int M, int N, int b, zc *G, zc *X, long long ldX, const zc *det, const zc *e1,
                    const zc *e2, zc *scal, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    epilogue_kernel<<<grid_for((long long)M * b * N), NT, 0, st>>>(M, N, b, G, X, ldX, det, e1, e2, scal);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

size_t accumulate_scratch_bytes(int nslot, int M, int N, int b) {
    const long long ngroups = (b + ACC_GROUP - 1) / ACC_GROUP;
    return (size_t)ngroups * ((size_t)nslot * M * N + nslot) * sizeof(AccPart);
}

int launch_accumulate(int nslot, int M, int N, int b, const zc *Wt, long long nomega, long long w0, const int *slotmap,
                      const zc *G, const zc *R, long long ldX, const zc *scal, zc *accG, zc *compG, zc *accR,
                      zc *compR, zc *accHS, zc *compHS, void *scratch, cudaStream_t st, int conj_weights) {
    const int ngroups = (b + ACC_GROUP - 1) / ACC_GROUP;
    AccPart *part = reinterpret_cast<AccPart *>(scratch);
    AccPart *part_hs = part + (size_t)ngroups * nslot * M * N;
    {
        ProfScope prof(st, PROF_MEMORY);
        accumulate_partial_kernel<<<grid_for((long long)ngroups * nslot * M * N), NT, 0, st>>>(
            nslot, M, N, b, Wt, nomega, w0, G, R, ldX, scal, ngroups, part, part_hs, conj_weights);
    }
    ++g_launches;
    PHF_CHECK_LAUNCH();
    {
        ProfScope prof(st, PROF_MEMORY);
        accumulate_final_kernel<<<grid_for((long long)nslot * M * N), NT, 0, st>>>(
            nslot, M, N, slotmap, ngroups, part, part_hs, accG, compG, accR, compR, accHS, compHS);
    }
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_ket_prep(int M, int N, int b, const zc *Hb, const zc *bra, const zc *e1, const zc *e2, zc *V, long long ld,
                    cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    ket_prep_kernel<<<grid_for((long long)M * b * N), NT, 0, st>>>(M, N, b, Hb, bra, e1, e2, V, ld);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_scale_conj_det(int M, int N, int b, const zc *det, zc *P, long long ld, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    scale_conj_det_kernel<<<grid_for((long long)M * b * N), NT, 0, st>>>(M, N, b, det, P, ld);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_average(long long n, const zc *a, const zc *b, zc *out, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    average_kernel<<<grid_for(n), NT, 0, st>>>(n, a, b, out);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_fold_comp(long long n, zc *a, const zc *c, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    fold_comp_kernel<<<grid_for(n), NT, 0, st>>>(n, a, c);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_permute_h2(int M, const zc *H2, zc *H2r, cudaStream_t st) {
    long long tot = (long long)M * M * M * M;
    ProfScope prof(st, PROF_MEMORY);
    permute_h2_kernel<<<grid_for(tot), NT, 0, st>>>(M, H2, H2r);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_permute_rows(int M, int N, int nbatch, const int *rowmap, const zc *in, long long ldin, long long bs_in,
                        zc *out, long long bs_out, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    permute_rows_kernel<<<dim3(grid_for((long long)M * N), nbatch), NT, 0, st>>>(M, N, rowmap, in, ldin, bs_in, out,
                                                                                 bs_out);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_gather_p(int n, int b, const zc *rho, zc *P, long long ldp, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    gather_p_kernel<<<grid_for((long long)n * n * b), NT, 0, st>>>(n, b, rho, P, ldp);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_gather_kin(int n, int b, const zc *rho, zc *Kin, long long ldk, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    gather_kin_kernel<<<grid_for((long long)n * n * b * 4), NT, 0, st>>>(n, b, rho, Kin, ldk);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_spin_block_y(int n, int N, int bc, int w0, int blk, const zc *R1b, const zc *T2, long long ld2, zc *Ys,
                        long long ld, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    spin_block_y_kernel<<<grid_for(2LL * n * bc * N), NT, 0, st>>>(n, N, bc, w0, blk, R1b, T2, ld2, Ys, ld);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_add_coulomb_diag(int n, int b, const double *Jr, long long jrs, long long jcs, zc *Gam, cudaStream_t st,
                            const double *h) {
    ProfScope prof(st, PROF_MEMORY);
    add_coulomb_diag_kernel<<<grid_for(2LL * n * n * b), NT, 0, st>>>(n, b, Jr, jrs, jcs, Gam, h);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

// out (2M x 2N): rows 2j and 2j + 1 of the real operand of rho = X bra^H (see launch_bra_rho_operand)
__global__ void bra_rho_operand_kernel(int M, int N, const zc *bra, double *out) {
    const long long total = (long long)M * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / N), k = (int)(e - (long long)j * N);
        const zc b = bra[e];
        double *r0 = out + (long long)(2 * j) * (2 * N) + 2 * k, *r1 = r0 + 2 * N;
        r0[0] = b.x;
        r0[1] = b.y;
        r1[0] = -b.y;
        r1[1] = b.x;
    }
}

int launch_bra_rho_operand(int M, int N, const zc *bra, double *out, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    bra_rho_operand_kernel<<<grid_for((long long)M * N), NT, 0, st>>>(M, N, bra, out);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_ek_sym_panel(int n, int i0, int ipanel, int k0, const int *pairs, const double *G, long long ldg,
                        double *EKs, double *EKa, cudaStream_t st) {
    const long long rows_s = (long long)ipanel * (n - i0) - (long long)ipanel * (ipanel - 1) / 2;
    if (n < 1 || n > 65535 || i0 < 0 || ipanel < 1 || i0 + ipanel > n || k0 < 0 || k0 > i0 ||
        ldg < ((long long)n - k0) * n) {
        set_error(PHF_ERR_ARG, "launch_ek_sym_panel: panel outside the index range or a short Gram block");
        return PHF_ERR_ARG;
    }
    const long long nn = n, t0 = (long long)i0 * nn - (long long)i0 * (i0 - 1) / 2;
    ProfScope prof(st, PROF_MEMORY);
    ek_sym_panel_kernel<<<(unsigned)rows_s, 256, 0, st>>>(n, i0, k0, pairs, t0, G, ldg, EKs, EKa);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_gather_kin_sym(int n, int b, const int *pairs, const zc *rho, zc *Kin, long long ldk, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    gather_kin_sym_kernel<<<grid_for((long long)n * (n + 1) / 2 * b * 4), NT, 0, st>>>(n, b, pairs, rho, Kin, ldk);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_ek_panel(int n, int ipanel, const double *G, long long ldg, double *EKp, long long lde, cudaStream_t st) {
    ProfScope prof(st, PROF_MEMORY);
    ek_panel_kernel<<<(unsigned)((long long)ipanel * n), NT, 0, st>>>(n, G, ldg, EKp, lde);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

int launch_assemble_gamma(int n, int b, const zc *J, long long ldj, const double *Jr, long long jrs, long long jcs,
                          const zc *Kc, long long ldk, const double *Kr, long long krs, long long kcs, zc *Gam,
                          cudaStream_t st, int ksym, const double *h) {
    ProfScope prof(st, PROF_MEMORY);
    assemble_gamma_kernel<<<grid_for(4LL * n * n * b), NT, 0, st>>>(n, b, J, ldj, Jr, jrs, jcs, Kc, ldk, Kr, krs, kcs,
                                                                    Gam, ksym, h);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

}  // namespace phf
