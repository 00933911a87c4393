// BuildSC on the GPU: the grid-projected product of a coupled-cluster-shaped vector (c0, c1, c2)
// with the projection operator, as the reference's linear-dependency solver uses it (LinDep.py:71-76,
// PHF_fort/PHFTools.f90:464-537, PHF_fort/BuildSC_dr.f90).  Per grid point w = (il, iy, ipg):
//
//   R_w = R1[il] R2[iy] Rpg[ipg];   S_w = R_w[:N, :N];   Y_w = [R_w[:, :N] S_w^-1 | 0]   (RDM of [I; 0])
//   c1_w = R_w c1 R_w^H;   c2_w = c2 with every index transformed by R_w^H              (ao2mo2, ao2mo4)
//   (a0, a1, a2)_w = BuildSC_Vec(c0, c1_w, c2_w, Y_w)                                   (BuildSC_dr.f90)
//   t += weightsp(il, iy) det S_w wpg(ipg) (sum conj fsp)(sum fsp) a_w,   ovlp likewise;   t /= ovlp
//
// with wpg(ipg) = sum_pq weightpg(ipg, p, q) conj(fpg_p) fpg_q (the Wigner factor of :516 is set to one
// at :518 in the reference, and so here).  Points run in chunks of b: every tensor of a chunk is
// batched over its points, the M^5 contractions (ao2mo4 and the four-index products of BuildSC_Vec)
// are strided batched FP64 GEMMs on the tensor cores (zgemm_strided), the M^4 index permutations,
// outer products and two-index contractions are the elementwise kernels below.  Tensors follow the
// Fortran arrays: X(a, b, c, d) at a + M b + M^2 c + M^3 d, X(a, b) at a + M b.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "phf_internal.h"

namespace phf {
namespace {

constexpr int NT = 256;

inline int blocks_for(long long n) {
    long long g = (n + NT - 1) / NT;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

// Strides of a four-index operand over the output's loop indices (a, b, c, d) and the point.
struct S4 {
    long long s[4];
    long long w;
};

// out(a,b,c,d)_w = [init ? 0 : out] + sign alpha_w in(.)_w   (alpha: per-point scalars or nullptr = 1)
__global__ void axpy4_kernel(int n0, int n1, int n2, int n3, int b, zc *out, S4 os, const zc *in, S4 is,
                             const zc *alpha, double sign, int init) {
    const long long tot = (long long)n0 * n1 * n2 * n3 * b;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        long long r = e;
        const int a = (int)(r % n0); r /= n0;
        const int bb = (int)(r % n1); r /= n1;
        const int c = (int)(r % n2); r /= n2;
        const int d = (int)(r % n3);
        const long long w = r / n3;
        const long long io = a * is.s[0] + bb * is.s[1] + c * is.s[2] + d * is.s[3] + w * is.w;
        const long long oo = a * os.s[0] + bb * os.s[1] + c * os.s[2] + d * os.s[3] + w * os.w;
        zc v = sign * in[io];
        if (alpha) v = alpha[w] * v;
        out[oo] = init ? v : out[oo] + v;
    }
}

// out(a,b,c,d)_w = [init ? 0 : out] + sign alpha_w X(.)_w Z(.)_w   (X and Z each use two of the indices)
__global__ void outer4_kernel(int M, int b, zc *out, const zc *X, S4 xs, const zc *Z, S4 zs, const zc *alpha,
                              double sign, int init) {
    const long long M4 = (long long)M * M * M * M, tot = M4 * b;
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < tot; e += (long long)gridDim.x * NT) {
        const long long w = e / M4, r = e - w * M4;
        const int a = (int)(r % M), bb = (int)((r / M) % M), c = (int)((r / ((long long)M * M)) % M),
                  d = (int)(r / ((long long)M * M * M));
        const zc x = X[a * xs.s[0] + bb * xs.s[1] + c * xs.s[2] + d * xs.s[3] + w * xs.w];
        const zc z = Z[a * zs.s[0] + bb * zs.s[1] + c * zs.s[2] + d * zs.s[3] + w * zs.w];
        zc v = sign * (x * z);
        if (alpha) v = alpha[w] * v;
        out[e] = init ? v : out[e] + v;
    }
}

// out(a, b)_w = [init ? 0 : out] + sign sum_{c,d} Y(c, d)_w T(a, b, c, d)_w  (T read with strides ts)
__global__ void contract2_kernel(int M, zc *out, const zc *Y, const zc *T, S4 ts, double sign, int init) {
    __shared__ zc sh[NT];
    const int a = blockIdx.x % M, bb = blockIdx.x / M;
    const long long w = blockIdx.y;
    const zc *y = Y + w * (long long)M * M;
    const zc *t = T + w * ts.w + a * ts.s[0] + bb * ts.s[1];
    zc acc = mkz(0, 0);
    for (int e = threadIdx.x; e < M * M; e += NT) {
        const int c = e % M, d = e / M;
        acc = acc + y[c + (long long)M * d] * t[c * ts.s[2] + d * ts.s[3]];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        zc *o = out + w * (long long)M * M + a + (long long)M * bb;
        const zc v = sign * sh[0];
        *o = init ? v : *o + v;
    }
}

// out_w = [init ? 0 : out_w] + sign sum_{a,b} X(a, b)_w Z(.)_w  (X plain M x M, Z with strides zs over (a, b))
__global__ void trace2_kernel(int M, zc *out, const zc *X, const zc *Z, long long za, long long zb, long long zw,
                              double sign, int init) {
    __shared__ zc sh[NT];
    const long long w = blockIdx.x;
    zc acc = mkz(0, 0);
    for (int e = threadIdx.x; e < M * M; e += NT) {
        const int a = e % M, bb = e / M;
        acc = acc + X[w * (long long)M * M + e] * Z[w * zw + a * za + bb * zb];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[w] = init ? sign * sh[0] : out[w] + sign * sh[0];
}

// per point: scalar out_w = [init ? 0 : out_w] + x_w (+ c when given)
__global__ void scalar_kernel(int b, zc *out, const zc *x, zc c, int init) {
    const int w = blockIdx.x * NT + threadIdx.x;
    if (w >= b) return;
    const zc v = (x ? x[w] : mkz(0, 0)) + c;
    out[w] = init ? v : out[w] + v;
}

// weight of point w: det S_w weightsp(il, iy) wpg(ipg) fsum; overlap sum in fixed order by one thread
__global__ void weights_kernel(int b, int w0, const zc *det, const zc *wt, zc *sc, zc *ovlp) {
    const int w = blockIdx.x * NT + threadIdx.x;
    if (w < b) sc[w] = det[w] * wt[w0 + w];
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        zc s = *ovlp;
        for (int i = 0; i < b; ++i) s = s + det[i] * wt[w0 + i];
        *ovlp = s;
    }
}

// acc[e] += sum_w t_w[e] sc_w over the chunk's points, in point order (n elements per point)
__global__ void accumulate_kernel(long long n, int b, const zc *t, const zc *sc, zc *acc) {
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < n; e += (long long)gridDim.x * NT) {
        zc s = acc[e];
        for (int w = 0; w < b; ++w) s = s + t[w * n + e] * sc[w];
        acc[e] = s;
    }
}

const zc ONE{1.0, 0.0}, ZERO{0.0, 0.0}, MONE{-1.0, 0.0};

View V(const zc *p, long long rs, long long cs, long long bs0 = 0, long long bs1 = 0, int conj = 0) {
    View v;
    v.p = p;
    v.rs = rs;
    v.cs = cs;
    v.bs0 = bs0;
    v.bs1 = bs1;
    v.conj = conj;
    v.real = 0;
    return v;
}
OutView O(zc *p, long long rs, long long cs, long long bs0 = 0, long long bs1 = 0) {
    OutView o;
    o.p = p;
    o.rs = rs;
    o.cs = cs;
    o.bs0 = bs0;
    o.bs1 = bs1;
    return o;
}

// Launch helpers over a chunk of b points (M, b captured in a small context).
struct Ctx {
    int M, b;
    cudaStream_t st;
    long long M2() const { return (long long)M * M; }
    long long M3() const { return (long long)M * M * M; }
    long long M4() const { return M2() * M2(); }
    // index-permuted read of a four-index tensor: in(p[0], p[1], p[2], p[3]) with p a permutation of
    // the output's (a, b, c, d) -- e.g. "bacd" reads in(b, a, c, d)
    S4 perm(const char *p) const {
        S4 s{{0, 0, 0, 0}, M4()};
        const long long str[4] = {1, (long long)M, M2(), M3()};
        for (int pos = 0; pos < 4; ++pos) s.s[p[pos] - 'a'] += str[pos];
        return s;
    }
    // a two-index operand X(i, j) over the output's loop indices: i, j name which of a..d
    S4 two(char i, char j) const {
        S4 s{{0, 0, 0, 0}, M2()};
        s.s[i - 'a'] += 1;
        s.s[j - 'a'] += M;
        return s;
    }
    int axpy4(zc *out, const zc *in, const char *p, double sign, int init, const zc *alpha = nullptr) const {
        S4 os{{1, M, M2(), M3()}, M4()};
        axpy4_kernel<<<blocks_for(M4() * b), NT, 0, st>>>(M, M, M, M, b, out, os, in, perm(p), alpha, sign, init);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    // two-index axpy: out(a, b) (+)= sign alpha in(a, b) or in(b, a) (transposed)
    int axpy2(zc *out, const zc *in, bool transposed, double sign, int init, const zc *alpha = nullptr) const {
        S4 os{{1, M, 0, 0}, M2()};
        S4 is{{transposed ? M : 1, transposed ? 1 : M, 0, 0}, M2()};
        axpy4_kernel<<<blocks_for(M2() * b), NT, 0, st>>>(M, M, 1, 1, b, out, os, in, is, alpha, sign, init);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    int outer4(zc *out, const zc *X, S4 xs, const zc *Z, S4 zs, double sign, int init,
               const zc *alpha = nullptr) const {
        outer4_kernel<<<blocks_for(M4() * b), NT, 0, st>>>(M, b, out, X, xs, Z, zs, alpha, sign, init);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    // out(a, b) (+)= sign sum_{c,d} Y(c, d) T(q) with q the index order of T over (a, b, c, d)
    int contract2(zc *out, const zc *Y, const zc *T, const char *q, double sign, int init) const {
        contract2_kernel<<<dim3((unsigned)(M * M), (unsigned)b), NT, 0, st>>>(M, out, Y, T, perm(q), sign, init);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    // out_w (+)= sign sum_{a,b} X(a, b) Z(a, b) or Z(b, a)
    int trace2(zc *out, const zc *X, const zc *Z, bool transposed, double sign, int init) const {
        trace2_kernel<<<b, NT, 0, st>>>(M, out, X, Z, transposed ? M : 1, transposed ? 1 : M, M2(), sign, init);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        return PHF_OK;
    }
    // two-index product C(a, b) = alpha sum_c A(., .) B(., .) + beta C with the views' strides
    int gemm2(zc *C, const View &A, const View &B, zc alpha = ONE, zc beta = ZERO) const {
        return zgemm_strided(M, M, M, b, 1, alpha, A, B, beta, O(C, 1, M, M2()), nullptr, st);
    }
    // four-index product T(a, b, c, d) = alpha sum_e Y(e, a) or Y(a, e) (transposed) times X(b, c, d, e)
    // + beta T: a strided GEMM with rows (b, c, d) and columns a
    int gemm4(zc *T, const zc *Y, bool y_ae, const zc *X, zc alpha = ONE, zc beta = ZERO) const {
        const View A = V(X, 1, M3(), M4());
        const View B = y_ae ? V(Y, M, 1, M2()) : V(Y, 1, M, M2());
        return zgemm_strided((int)M3(), M, M, b, 1, alpha, A, B, beta, O(T, M, 1, M4()), nullptr, st);
    }
};

}  // namespace

// BuildSC (PHF_fort/PHFTools.f90:464-537).  Host arrays in the reference's Fortran layouts.
int buildsc_run(phf_complex c0h, const phf_complex *c1h, const phf_complex *c2h, int nocc, int nso, const int *ngrid,
                int npg, const phf_complex *r1h, const phf_complex *r2h, const phf_complex *rpgh,
                const double *weightsp, const double *weightpg, int ncisp, int ncipg, const phf_complex *fsp,
                const phf_complex *fpg, size_t workspace, phf_complex *t0h, phf_complex *t1h, phf_complex *t2h) {
    const int M = nso, N = nocc, nl = ngrid[0], ny = ngrid[1];
    const long long M2 = (long long)M * M, M4 = M2 * M2;
    const int nw = nl * ny * npg;
    // per-point weight factor weightsp(il, iy) wpg(ipg) (sum conj fsp)(sum fsp)
    cd fs = 0, fsc = 0;
    for (int m = 0; m < ncisp; ++m) {
        fs += cd(fsp[m].re, fsp[m].im);
        fsc += std::conj(cd(fsp[m].re, fsp[m].im));
    }
    std::vector<cd> wt(nw);
    for (int il = 0; il < nl; ++il)
        for (int iy = 0; iy < ny; ++iy)
            for (int ig = 0; ig < npg; ++ig) {
                cd wpg = 0;
                for (int p = 0; p < ncipg; ++p)
                    for (int q = 0; q < ncipg; ++q)
                        wpg += weightpg[(size_t)ig + (size_t)npg * ((size_t)p + (size_t)ncipg * q)] *
                               std::conj(cd(fpg[p].re, fpg[p].im)) * cd(fpg[q].re, fpg[q].im);
                wt[((size_t)il * ny + iy) * npg + ig] = weightsp[(size_t)il + (size_t)nl * iy] * wpg * fsc * fs;
            }
    // chunk from the workspace budget: eight M^4 and about twenty M^2 tensors per point
    const size_t per = (8 * (size_t)M4 + 24 * (size_t)M2 + (size_t)N * N + 16) * sizeof(zc);
    const size_t budget = workspace ? workspace : ((size_t)4 << 30);
    const int b = (int)std::max<size_t>(1, std::min<size_t>(budget / per, (size_t)nw));

    Arena ar;
    zc *R1 = nullptr, *R2 = nullptr, *Rpg = nullptr, *c1 = nullptr, *c2 = nullptr, *wtd = nullptr;
    long long *offs = nullptr;
    // rotations column-major per index: R(i, j) at i + M j
    auto rot = [&](const phf_complex *src, int cnt, zc **dst) -> int {
        PHF_TRY(ar.alloc(dst, (size_t)cnt * M2));
        std::vector<zc> h((size_t)cnt * M2);
        for (int g = 0; g < cnt; ++g)
            for (int j = 0; j < M; ++j)
                for (int i = 0; i < M; ++i) {
                    const phf_complex v = src[(size_t)g + (size_t)cnt * ((size_t)i + (size_t)M * j)];
                    h[(size_t)g * M2 + i + (size_t)M * j] = zc{v.re, v.im};
                }
        PHF_CUDA(cudaMemcpy(*dst, h.data(), h.size() * sizeof(zc), cudaMemcpyHostToDevice));
        return PHF_OK;
    };
    PHF_TRY(rot(r1h, nl, &R1));
    PHF_TRY(rot(r2h, ny, &R2));
    PHF_TRY(rot(rpgh, npg, &Rpg));
    PHF_TRY(ar.alloc(&c1, (size_t)M2));
    PHF_TRY(ar.alloc(&c2, (size_t)M4));
    PHF_CUDA(cudaMemcpy(c1, c1h, M2 * sizeof(zc), cudaMemcpyHostToDevice));
    PHF_CUDA(cudaMemcpy(c2, c2h, M4 * sizeof(zc), cudaMemcpyHostToDevice));
    PHF_TRY(ar.alloc(&wtd, (size_t)nw));
    PHF_CUDA(cudaMemcpy(wtd, wt.data(), nw * sizeof(zc), cudaMemcpyHostToDevice));
    // GEMM offsets: T_w = R2[iy] Rpg[ipg], then R_w = R1[il] T_w
    std::vector<long long> o1(3 * (size_t)nw), o2(3 * (size_t)nw);
    for (int w = 0; w < nw; ++w) {
        const int il = w / (ny * npg), iy = (w / npg) % ny, ig = w % npg;
        o1[3 * w] = (long long)iy * M2;
        o1[3 * w + 1] = (long long)ig * M2;
        o1[3 * w + 2] = 0;
        o2[3 * w] = (long long)il * M2;
        o2[3 * w + 1] = 0;
        o2[3 * w + 2] = 0;
    }
    PHF_TRY(ar.alloc(&offs, 6 * (size_t)nw));
    PHF_CUDA(cudaMemcpy(offs, o1.data(), o1.size() * sizeof(long long), cudaMemcpyHostToDevice));
    PHF_CUDA(cudaMemcpy(offs + 3 * (size_t)nw, o2.data(), o2.size() * sizeof(long long), cudaMemcpyHostToDevice));

    // chunk workspace
    zc *T = nullptr, *R = nullptr, *Sinv = nullptr, *det = nullptr, *logdet = nullptr, *Y = nullptr, *c1t = nullptr,
       *t2d = nullptr, *sc = nullptr, *sclr = nullptr, *acc0 = nullptr, *acc1 = nullptr, *acc2 = nullptr,
       *ovlp = nullptr;
    zc *B4[7] = {};
    zc *B2[18] = {};
    int *flag = nullptr;
    PHF_TRY(ar.alloc(&T, (size_t)b * M2));
    PHF_TRY(ar.alloc(&R, (size_t)b * M2));
    PHF_TRY(ar.alloc(&Sinv, (size_t)b * N * N));
    PHF_TRY(ar.alloc(&det, (size_t)b));
    PHF_TRY(ar.alloc(&logdet, (size_t)b));
    PHF_TRY(ar.alloc(&Y, (size_t)b * M2));
    PHF_TRY(ar.alloc(&c1t, (size_t)b * M2));
    PHF_TRY(ar.alloc(&t2d, (size_t)b * M2));
    PHF_TRY(ar.alloc(&sc, (size_t)b));
    PHF_TRY(ar.alloc(&sclr, 4 * (size_t)b));
    for (auto &p : B4) PHF_TRY(ar.alloc(&p, (size_t)b * M4));
    for (auto &p : B2) PHF_TRY(ar.alloc(&p, (size_t)b * M2));
    PHF_TRY(ar.alloc(&acc0, 1));
    PHF_TRY(ar.alloc(&acc1, (size_t)M2));
    PHF_TRY(ar.alloc(&acc2, (size_t)M4));
    PHF_TRY(ar.alloc(&ovlp, 1));
    PHF_TRY(ar.alloc(&flag, 1));
    cudaStream_t st = 0;
    PHF_CUDA(cudaMemsetAsync(acc0, 0, sizeof(zc), st));
    PHF_CUDA(cudaMemsetAsync(acc1, 0, M2 * sizeof(zc), st));
    PHF_CUDA(cudaMemsetAsync(acc2, 0, M4 * sizeof(zc), st));
    PHF_CUDA(cudaMemsetAsync(ovlp, 0, sizeof(zc), st));
    PHF_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
    // four-index buffers (reused as the sequence allows) and two-index intermediates
    zc *c2t = B4[0], *tau11 = B4[0], *tmp = B4[1], *tau9 = B4[1], *tau19 = B4[1], *tau0 = B4[2], *tau10 = B4[3],
       *tau16 = B4[4], *tau22 = B4[5], *a2 = B4[6];
    zc *tau1 = B2[0], *tau2 = B2[1], *tau5 = B2[2], *tau6 = B2[3], *tau7 = B2[4], *tau13 = B2[5], *tau14 = B2[6],
       *tau15 = B2[7], *tau17 = B2[8], *tau18 = B2[9], *tau21 = B2[10], *tau24 = B2[11], *tau25 = B2[12],
       *tau26 = B2[13], *tau27 = B2[14], *a1 = B2[15];
    zc *tau3 = sclr, *tau8 = sclr + b, *tau23 = sclr + 2 * (size_t)b, *a0 = sclr + 3 * (size_t)b;
    const zc c0{c0h.re, c0h.im};

    for (int w0 = 0; w0 < nw; w0 += b) {
        const int bc = std::min(b, nw - w0);
        const Ctx x{M, bc, st};
        const long long M3 = x.M3();
        // R_w = R1[il] (R2[iy] Rpg[ipg])
        PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, V(R2, 1, M), V(Rpg, 1, M), ZERO, O(T, 1, M, M2), offs + 3LL * w0,
                              st));
        PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, V(R1, 1, M), V(T, 1, M, M2), ZERO, O(R, 1, M, M2),
                              offs + 3LL * nw + 3LL * w0, st));
        // RDM of [I; 0]: S = R[:N, :N] (read transposed, so the row-major inverse is S^-1 column-major)
        PHF_TRY(overlap_inverse(N, bc, R, M, M2, Sinv, N, (long long)N * N, det, logdet, flag, st));
        PHF_CUDA(cudaMemsetAsync(Y, 0, (size_t)bc * M2 * sizeof(zc), st));
        PHF_TRY(zgemm_strided(M, N, N, bc, 1, ONE, V(R, 1, M, M2), V(Sinv, 1, N, (long long)N * N), ZERO,
                              O(Y, 1, M, M2), nullptr, st));
        // c1_w = R c1 R^H (ao2mo2 with R^H)
        PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, V(R, 1, M, M2), V(c1, 1, M), ZERO, O(t2d, 1, M, M2), nullptr, st));
        PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, V(t2d, 1, M, M2), V(R, M, 1, M2, 0, 1), ZERO, O(c1t, 1, M, M2),
                              nullptr, st));
        // c2_w = ao2mo4(c2, U = R^H), U(x, l) = conj(R(l, x)): four one-index transforms
        PHF_TRY(zgemm_strided((int)M3, M, M, bc, 1, ONE, V(c2, 1, M3, 0), V(R, M, 1, M2, 0, 1), ZERO,
                              O(tmp, 1, M3, M4), nullptr, st));  // tmp(p,q,r,l) = sum_x U(x,l) c2(p,q,r,x)
        PHF_TRY(zgemm_strided((int)M2, M, M, M, bc, ONE, V(tmp, 1, M2, M3, M4), V(R, M, 1, 0, M2, 1), ZERO,
                              O(c2t, 1, M2, M3, M4), nullptr, st));  // (p,q,k,l) = sum_x U(x,k) tmp(p,q,x,l)
        PHF_TRY(zgemm_strided(M, M, M, (int)M2, bc, ONE, V(c2t, 1, M, M2, M4), V(R, M, 1, 0, M2), ZERO,
                              O(tmp, 1, M, M2, M4), nullptr, st));  // (p,j,k,l) = sum_x conj U(x,j) (p,x,k,l)
        PHF_TRY(zgemm_strided(M, (int)M3, M, bc, 1, ONE, V(R, 1, M, M2), V(tmp, 1, M, M4), ZERO, O(c2t, 1, M, M4),
                              nullptr, st));  // (i,j,k,l) = sum_x conj U(x,i) (x,j,k,l)

        // ---- BuildSC_Vec (PHF_fort/BuildSC_dr.f90), Y = the transition density of each point
        PHF_TRY(x.axpy4(tau0, c2t, "abcd", 1.0, 1));
        PHF_TRY(x.axpy4(tau0, c2t, "bacd", -1.0, 0));
        PHF_TRY(x.contract2(tau1, Y, tau0, "dabc", 1.0, 1));                 // tau1 = Y(c,d) tau0(d,a,b,c)
        PHF_TRY(x.axpy2(tau2, tau1, false, -1.0, 1));
        PHF_TRY(x.axpy2(tau6, tau1, false, -1.0, 1));
        PHF_TRY(x.trace2(tau8, Y, tau1, true, -1.0, 1));                      // tau8 = -Y(a,b) tau1(b,a)
        PHF_TRY(x.outer4(a2, Y, x.two('a', 'c'), Y, x.two('b', 'd'), 1.0, 1, tau8));
        PHF_TRY(x.outer4(a2, Y, x.two('a', 'd'), Y, x.two('b', 'c'), -1.0, 0, tau8));
        PHF_TRY(x.axpy2(tau13, tau1, false, -1.0, 1));
        PHF_TRY(x.contract2(tau5, Y, tau0, "adcb", 1.0, 1));                 // tau5 = Y(c,d) tau0(a,d,c,b)
        PHF_TRY(x.axpy2(tau6, tau5, false, -1.0, 0));
        PHF_TRY(x.axpy2(tau13, tau5, false, -1.0, 0));
        PHF_TRY(x.gemm2(tau14, V(Y, 1, M, M2), V(tau13, 1, M, M2)));         // Y(a,c) tau13(c,b)
        PHF_TRY(x.gemm2(tau15, V(Y, M, 1, M2), V(tau14, M, 1, M2)));         // Y(c,a) tau14(b,c)
        PHF_TRY(x.outer4(tau16, Y, x.two('a', 'c'), tau15, x.two('d', 'b'), -1.0, 1));
        PHF_TRY(x.gemm2(tau21, V(Y, M, 1, M2), V(tau13, M, 1, M2)));         // Y(c,a) tau13(b,c)
        PHF_TRY(x.outer4(tau22, Y, x.two('a', 'b'), tau21, x.two('c', 'd'), 1.0, 1));
        PHF_TRY(x.axpy2(tau2, c1t, false, 1.0, 0));
        PHF_TRY(x.trace2(tau3, Y, tau2, true, 1.0, 1));                       // tau3 = Y(a,b) tau2(b,a)
        PHF_TRY(x.axpy2(a1, Y, false, 1.0, 1, tau3));                         // t1 = tau3 Y
        // tau4 = -tau0, so tau7 = -Y.tau4(d,a,b,c) - Y.tau4(a,d,c,b) = tau1 + tau5 (sign flips are exact)
        PHF_TRY(x.axpy2(tau7, tau1, false, 1.0, 1));
        PHF_TRY(x.axpy2(tau7, tau5, false, 1.0, 0));
        PHF_TRY(x.axpy2(tau6, c1t, false, 1.0, 0));
        PHF_TRY(x.gemm2(tau7, V(Y, 1, M, M2), V(tau6, 1, M, M2), ONE, ONE));  // + Y(a,c) tau6(c,b)
        PHF_TRY(x.axpy2(tau7, c1t, false, -1.0, 0));
        PHF_TRY(x.gemm2(a1, V(tau7, 1, M, M2), V(Y, 1, M, M2), MONE, ONE));  // - Y(c,b) tau7(a,c)
        PHF_TRY(x.gemm4(tau9, Y, false, c2t));                                // Y(e,a) c2(b,c,d,e)
        PHF_TRY(x.gemm4(tau10, Y, false, tau9));                              // Y(e,a) tau9(b,c,d,e)
        PHF_TRY(x.gemm4(tau11, Y, true, tau10));                              // Y(a,e) tau10(b,c,d,e)
        PHF_TRY(x.gemm4(tau16, Y, true, tau11, ONE, ONE));                    // + tau12 = Y(a,e) tau11(b,c,d,e)
        PHF_TRY(x.axpy4(a2, tau16, "abcd", 1.0, 0));
        PHF_TRY(x.axpy4(a2, tau16, "abdc", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau16, "bacd", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau16, "badc", 1.0, 0));
        PHF_TRY(x.axpy4(tau19, tau10, "abcd", -1.0, 1));
        PHF_TRY(x.axpy4(tau19, tau10, "abdc", 1.0, 0));
        PHF_TRY(x.gemm4(tau22, Y, true, tau19, MONE, ONE));                   // - tau20 = Y(a,e) tau19(b,c,d,e)
        PHF_TRY(x.axpy4(a2, tau22, "acdb", 1.0, 0));
        PHF_TRY(x.axpy4(a2, tau22, "adcb", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau22, "bcda", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau22, "bdca", 1.0, 0));
        PHF_TRY(x.axpy4(a2, tau10, "cdab", 1.0, 0));
        PHF_TRY(x.axpy4(a2, tau10, "cdba", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau10, "dcab", -1.0, 0));
        PHF_TRY(x.axpy4(a2, tau10, "dcba", 1.0, 0));
        PHF_TRY(x.gemm2(tau17, V(Y, M, 1, M2), V(c1t, M, 1, M2)));           // Y(c,a) c1(b,c)
        PHF_TRY(x.gemm2(tau18, V(Y, 1, M, M2), V(tau17, M, 1, M2)));         // Y(a,c) tau17(b,c)
        PHF_TRY(x.outer4(a2, Y, x.two('a', 'c'), tau18, x.two('b', 'd'), -1.0, 0));
        PHF_TRY(x.outer4(a2, Y, x.two('b', 'c'), tau18, x.two('a', 'd'), 1.0, 0));
        PHF_TRY(x.outer4(a2, Y, x.two('a', 'c'), tau17, x.two('d', 'b'), 1.0, 0));
        PHF_TRY(x.outer4(a2, Y, x.two('b', 'c'), tau17, x.two('d', 'a'), -1.0, 0));
        PHF_TRY(x.trace2(tau23, Y, c1t, true, 1.0, 1));                       // tau23 = Y(b,a) c1(a,b)
        PHF_TRY(x.axpy2(tau27, Y, true, 1.0, 1, tau23));                      // tau27 = tau23 Y(b,a)
        PHF_TRY(x.gemm2(tau24, V(Y, 1, M, M2), V(c1t, 1, M, M2)));           // Y(a,c) c1(c,b)
        PHF_TRY(x.axpy2(tau25, tau24, false, 1.0, 1));
        PHF_TRY(x.axpy2(tau25, c1t, false, -1.0, 0));
        PHF_TRY(x.gemm2(tau26, V(Y, M, 1, M2), V(tau25, M, 1, M2)));         // Y(c,a) tau25(b,c)
        PHF_TRY(x.axpy2(tau27, tau26, false, -1.0, 0));
        {
            // tau27 += c0 Y(b,a); t0 = tau3 + c0; t1 += c0 Y
            zc *c0w = sclr + 3 * (size_t)b;  // a0 holds c0 for every point first, then t0
            scalar_kernel<<<(bc + NT - 1) / NT, NT, 0, st>>>(bc, c0w, nullptr, c0, 1);
            ++g_launches;
            PHF_CHECK_LAUNCH();
            PHF_TRY(x.axpy2(tau27, Y, true, 1.0, 0, c0w));
            PHF_TRY(x.axpy2(a1, Y, false, 1.0, 0, c0w));
            scalar_kernel<<<(bc + NT - 1) / NT, NT, 0, st>>>(bc, a0, tau3, c0, 1);  // t0 = tau3 + c0
            ++g_launches;
            PHF_CHECK_LAUNCH();
        }
        PHF_TRY(x.outer4(a2, Y, x.two('b', 'd'), tau27, x.two('c', 'a'), 1.0, 0));
        PHF_TRY(x.outer4(a2, Y, x.two('a', 'd'), tau27, x.two('c', 'b'), -1.0, 0));

        // ---- weights and accumulation over the chunk's points (fixed order)
        weights_kernel<<<(bc + NT - 1) / NT, NT, 0, st>>>(bc, w0, det, wtd, sc, ovlp);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        accumulate_kernel<<<1, NT, 0, st>>>(1, bc, a0, sc, acc0);
        accumulate_kernel<<<blocks_for(M2), NT, 0, st>>>(M2, bc, a1, sc, acc1);
        accumulate_kernel<<<blocks_for(M4), NT, 0, st>>>(M4, bc, a2, sc, acc2);
        g_launches += 3;
        PHF_CHECK_LAUNCH();
    }
    std::vector<cd> h0(1), h1(M2), h2(M4), ho(1);
    int hflag = 0;
    PHF_CUDA(cudaMemcpyAsync(h0.data(), acc0, sizeof(zc), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaMemcpyAsync(h1.data(), acc1, M2 * sizeof(zc), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaMemcpyAsync(h2.data(), acc2, M4 * sizeof(zc), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaMemcpyAsync(ho.data(), ovlp, sizeof(zc), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaStreamSynchronize(st));
    if (hflag & 1) {
        set_error(PHF_ERR_SINGULAR, "BuildSC: a rotated overlap R[:N, :N] is exactly singular");
        return PHF_ERR_SINGULAR;
    }
    if (hflag & 2 || !std::isfinite(ho[0].real()) || ho[0] == cd(0, 0)) {
        set_error(PHF_ERR_NONFINITE, "BuildSC: non-finite or zero projected overlap");
        return PHF_ERR_NONFINITE;
    }
    const cd ov = ho[0];
    const cd v0 = h0[0] / ov;
    t0h->re = v0.real();
    t0h->im = v0.imag();
    for (long long i = 0; i < M2; ++i) {
        const cd v = h1[i] / ov;
        t1h[i].re = v.real();
        t1h[i].im = v.imag();
    }
    for (long long i = 0; i < M4; ++i) {
        const cd v = h2[i] / ov;
        t2h[i].re = v.real();
        t2h[i].im = v.imag();
    }
    return PHF_OK;
}

}  // namespace phf
