// Projected coupled-cluster grid kernel on the GPU: PbarHbarOlap (SUCCSD_Boson_cmplx/FPUCC.f90:14-272)
// with EvalKernel (:529-602) at every grid point, as the reference's PCC solver calls it once per
// Broyden iteration (Main.f90 PGCC -> BroydenIter).  Per grid point w = (il, iy, ipg):
//
//   R_w = R1[il] R2[iy] Rpg[ipg] (Rk(2) in the ncik = 2 pass)
//   (U0, U1)   = Thouless form of R_w [1; T1]                          ProjT1, FPUCC_Tools.f90:676-695
//   V = [1 0; -U1 1] R_w,  U' = T2 transformed by V (bra) and V^-1 (ket)   TransT2, PCCCI.f90:100-276
//   (C0, C1, C2) = second-order CI coefficients from U';  (W0, W1, W2) = CI2CC(C) (PCCCI.f90:72-98)
//   W0 <- W0 U0, W1 <- W1 + U1                                           DSTT2, FPUCC_Tools.f90:697-722
//   CCSD energy and residuals of (W1, W2) with the fixed Fock matrix and <pq||rs>  (CCRes.f90)
//   lambda and eps tensors of BuildKernSD (FPUCC_Tools.f90:291-436), times lambda0 = W0
//   sums += w_w (eps0, lambda0, eps1, lambda1, eps2, lambda2)      with w_w the Wigner x point-group weight
//
// Every tensor of a chunk of grid points is batched over its points.  Each contraction runs on this
// library's FP64 tensor-core GEMM (zgemm_strided): a small planner maps its index letters onto GEMM rows,
// columns, k and a batch index, choosing among the ways to group the letters the one whose strides let
// every operand be read in place (copying an operand into a contiguous order only when no grouping
// does), so a contraction is one batched GEMM launch over all points.  Index permutations, outer
// products and per-point scalings are one strided elementwise kernel.  Tensors are in the Fortran
// layouts (first index fastest), vo arrays (a, i) and vvoo arrays (a, b, i, j) with the virtual index
// relative to NOcc, NSO-sized arrays over the full range.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "phf_internal.h"

namespace phf {
namespace {

constexpr int NT = 256;
constexpr int MAXD = 6;

// device time of the grid pipeline of the last call (uploads excluded) and the FP64 flops its GEMMs ran
double g_pcc_ms = 0.0, g_pcc_flops = 0.0;
const zc ONE{1.0, 0.0}, ZERO{0.0, 0.0};

// ---------------------------------------------------------------- strided tensor views
// Element (i_0, .., i_{nd-1}) of grid point w at p + sum i_d st[d] + w ps (ps = 0: shared by all points).
struct TV {
    zc *p = nullptr;
    int nd = 0;
    int dim[MAXD] = {};
    long long st[MAXD] = {};
    long long ps = 0;
    int conj = 0;
};

TV tens(zc *p, std::initializer_list<int> dims, bool per_point = true) {
    TV t;
    t.p = p;
    long long s = 1;
    for (int d : dims) {
        t.dim[t.nd] = d;
        t.st[t.nd++] = s;
        s *= d;
    }
    t.ps = per_point ? s : 0;
    return t;
}

// sub-block at offsets `off`, sizes `n` of a view
TV blk(const TV &t, std::initializer_list<int> off, std::initializer_list<int> n) {
    TV r = t;
    int d = 0;
    for (int o : off) r.p += o * t.st[d++];
    d = 0;
    for (int k : n) r.dim[d++] = k;
    return r;
}

TV scal(zc *p, bool per_point = true) {
    TV t;
    t.p = p;
    t.ps = per_point ? 1 : 0;
    return t;
}

TV conjv(TV t) {
    t.conj ^= 1;
    return t;
}

long long numel(const TV &t) {
    long long n = 1;
    for (int d = 0; d < t.nd; ++d) n *= t.dim[d];
    return n;
}

inline int blocks_for(long long n) {
    long long g = (n + NT - 1) / NT;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

// ---------------------------------------------------------------- kernels
struct EwArgs {
    int nd;
    int dim[MAXD];
    long long cs[MAXD], as[MAXD], bs[MAXD];
    long long cps, aps, bps;
    zc *C;
    const zc *A, *B;
    int aconj, bconj;
    zc alpha, beta;
    long long per, total;
};

// C = beta C + alpha op(A) op(B) elementwise over a strided index space and the points (B optional)
__global__ void ew_kernel(EwArgs g) {
    const bool use_beta = (g.beta.x != 0.0 || g.beta.y != 0.0);
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < g.total; e += (long long)gridDim.x * NT) {
        const long long w = e / g.per;
        long long r = e - w * g.per;
        long long oc = w * g.cps, oa = w * g.aps, ob = w * g.bps;
        for (int d = 0; d < g.nd; ++d) {
            const long long i = r % g.dim[d];
            r /= g.dim[d];
            oc += i * g.cs[d];
            oa += i * g.as[d];
            ob += i * g.bs[d];
        }
        zc a = g.A[oa];
        if (g.aconj) a.y = -a.y;
        zc v = g.alpha * a;
        if (g.B) {
            zc b = g.B[ob];
            if (g.bconj) b.y = -b.y;
            v = v * b;
        }
        if (use_beta) v = v + g.beta * g.C[oc];
        g.C[oc] = v;
    }
}

// C(i, j)_w = beta C + alpha sum_s T(i, j, s)_w   (the partial products of a split-k GEMM, T contiguous)
__global__ void splitk_reduce_kernel(int m, int n, int S, long long total, const zc *T, OutView C, zc alpha,
                                     zc beta) {
    const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        const long long w = e / ((long long)m * n);
        const long long r = e - w * (long long)m * n;
        const int i = (int)(r % m), j = (int)(r / m);
        const zc *t = T + (w * S) * (long long)m * n + r;
        zc acc{0.0, 0.0};
        for (int q = 0; q < S; ++q) acc = acc + t[(long long)q * m * n];
        zc v = alpha * acc;
        zc *c = C.p + w * C.bs0 + i * C.rs + j * C.cs;
        if (use_beta) v = v + beta * *c;
        *c = v;
    }
}

// T[w S + s] = sum over the k-slice s of op(A)[k] op(B)[k]  (scalar contractions: one CTA per point and slice)
__global__ void dot_kernel(long long k, int S, View A, View B, zc *T) {
    __shared__ zc sh[NT];
    const long long w = blockIdx.x / S;
    const int s = (int)(blockIdx.x - w * S);
    const long long ks = (k + S - 1) / S, k0 = s * ks, k1 = (k0 + ks < k) ? k0 + ks : k;
    const zc *a = static_cast<const zc *>(A.p) + w * A.bs0;
    const zc *b = static_cast<const zc *>(B.p) + w * B.bs0;
    zc acc{0.0, 0.0};
    for (long long q = k0 + threadIdx.x; q < k1; q += NT) {
        zc x = a[q * A.cs], y = b[q * B.rs];
        if (A.conj) x.y = -x.y;
        if (B.conj) y.y = -y.y;
        acc = acc + x * y;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = NT / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) T[blockIdx.x] = sh[0];
}

// The (T) energy's triangular sum (CCSD_T_Ene, SUCCSD_Boson_cmplx/CCSD_T.f90:10-108) for one virtual
// triple a >= b >= c (blockIdx.x) of one grid point (blockIdx.y):
//   w = Perm3(W[abc] + W[cab] - W[bac]),  v = V[abc] + V[cab] - V[bac],
//   V[pqr](x,y,z) = W[pqr](x,y,z) + T1(p,x) <qr||yz> + f(p,x) T2(q,r,y,z)          (get_wv, :54-70)
//   part = sum_xyz w / (f_x + f_y + f_z - f_a - f_b - f_c) conj(v)
// with W[pqr](x,y,z) = sum_d <qr||dx> T2(p,d,y,z) - sum_l T2(q,r,x,l) <lp||yz> at W[x + o(q + v(r + v(p + v(y + o z))))]
// (the rows (x, q, r) of the GEMM that forms it, then its columns (p, y, z))
// and Perm3 w(x,y,z) = w(x,y,z) + w(z,x,y) + w(y,z,x).
struct TriplesArgs {
    int o, v;
    const int *tri;     // 3 per triple: a, b, c
    const zc *W;        // per point stride wps
    long long wps;
    const zc *T1;       // per point (v x o), stride t1ps
    long long t1ps;
    const zc *T2;       // per point (v, v, o, o), stride t2ps
    long long t2ps;
    const zc *vvoo;     // <ab||ij> view: strides 1, M, M^2, M^3
    const zc *fvo;      // F(o + a, i): strides 1, M
    const zc *fd;       // the Fock matrix F (M x M, column-major): its diagonal is read
    int M;
    zc *part;           // [point][triple]
    long long ntri;
};

__global__ void triples_kernel(TriplesArgs g) {
    __shared__ zc sh[NT];
    const long long t = blockIdx.x;
    const int w = blockIdx.y;
    const int o = g.o, v = g.v, M = g.M;
    const int a = g.tri[3 * t], b = g.tri[3 * t + 1], c = g.tri[3 * t + 2];
    const long long o3 = (long long)o * o * o, M2 = (long long)M * M;
    const zc *Wp = g.W + w * g.wps;
    const zc *t1 = g.T1 + w * g.t1ps, *t2 = g.T2 + w * g.t2ps;
    const int trip[3][3] = {{a, b, c}, {c, a, b}, {b, a, c}};
    const double sgn[3] = {1.0, 1.0, -1.0};
    long long base[3];
    for (int q = 0; q < 3; ++q) base[q] = (long long)o * (trip[q][1] + (long long)v * (trip[q][2] + (long long)v * trip[q][0]));
    const long long ov3 = (long long)o * v * v * v;
    const long long dg = M + 1;  // F(i, i) at fd[i (M + 1)]
    const zc eabc = g.fd[(o + a) * dg] + g.fd[(o + b) * dg] + g.fd[(o + c) * dg];
    zc acc{0.0, 0.0};
    for (int e = threadIdx.x; e < o3; e += NT) {
        const int x = e % o, y = (e / o) % o, z = e / (o * o);
        const long long e1 = x + ov3 * (y + (long long)o * z), e2 = z + ov3 * (x + (long long)o * y),
                        e3 = y + ov3 * (z + (long long)o * x);
        zc wv{0.0, 0.0}, vv{0.0, 0.0};
        for (int q = 0; q < 3; ++q) {
            const int p = trip[q][0], r1 = trip[q][1], r2 = trip[q][2];
            const zc *Wq = Wp + base[q];
            const zc w0 = Wq[e1];
            wv = wv + sgn[q] * (w0 + Wq[e2] + Wq[e3]);
            const zc extra = t1[p + (long long)v * x] * g.vvoo[r1 + M * (r2 + (long long)M * (y + (long long)M * z))] +
                             g.fvo[p + (long long)M * x] * t2[r1 + (long long)v * (r2 + (long long)v * (y + (long long)o * z))];
            vv = vv + sgn[q] * (w0 + extra);
        }
        const zc d = (g.fd[x * dg] + g.fd[y * dg] + g.fd[z * dg]) - eabc;
        acc = acc + divz(wv, d) * conjz(vv);
    }
    (void)M2;
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int h = NT / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) sh[threadIdx.x] = sh[threadIdx.x] + sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) g.part[w * g.ntri + t] = sh[0];
}

// The same sum without the W tensor (o <= kTriplesFusedMaxO): for its triple the CTA forms
//   S(x,y,z) = sum_q sgn_q W[pqr_q](x,y,z)   over the orders (abc), (cab), (bac), signs +, +, -,
// from <qr||dx>, T2 and <la||yz> directly into shared memory, then
//   w = S(x,y,z) + S(z,x,y) + S(y,z,x)  (Perm3 is linear),  v = S(x,y,z) + sum_q sgn_q (T1 <||> + f T2)_q.
constexpr int kTriplesFusedMaxO = 18;

__global__ void triples_fused_kernel(TriplesArgs g, const zc *vvvo, const zc *ovoo) {
    extern __shared__ zc Ssh[];
    __shared__ zc red[NT];
    const long long t = blockIdx.x;
    const int w = blockIdx.y;
    const int o = g.o, v = g.v, M = g.M;
    const int a = g.tri[3 * t], b = g.tri[3 * t + 1], c = g.tri[3 * t + 2];
    const int o3 = o * o * o;
    const long long M2 = (long long)M * M, M3 = M2 * M;
    const zc *t1 = g.T1 + w * g.t1ps, *t2 = g.T2 + w * g.t2ps;
    const int trip[3][3] = {{a, b, c}, {c, a, b}, {b, a, c}};
    const double sgn[3] = {1.0, 1.0, -1.0};
    const long long dg = M + 1;
    for (int e = threadIdx.x; e < o3; e += NT) {
        const int x = e % o, y = (e / o) % o, z = e / (o * o);
        zc acc{0.0, 0.0};
        for (int q = 0; q < 3; ++q) {
            const int p = trip[q][0], r1 = trip[q][1], r2 = trip[q][2];
            zc wq{0.0, 0.0};
            // sum_d <r1 r2||d x> T2(p, d, y, z)      (vvvo(r1, r2, d, x) at r1 + M r2 + M^2 d + M^3 x)
            const zc *vp = vvvo + r1 + (long long)M * r2 + M3 * x;
            const zc *tp = t2 + p + (long long)v * v * (y + (long long)o * z);
            for (int d = 0; d < v; ++d) wq = wq + vp[M2 * d] * tp[(long long)v * d];
            // - sum_l T2(r1, r2, x, l) <l p||y z>    (ovoo(l, p, y, z) at l + M p + M^2 y + M^3 z)
            const zc *sp = t2 + r1 + (long long)v * (r2 + (long long)v * x);
            const zc *op = ovoo + (long long)M * p + M2 * y + M3 * z;
            for (int l = 0; l < o; ++l) wq = wq - sp[(long long)v * v * o * l] * op[l];
            acc = acc + sgn[q] * wq;
        }
        Ssh[e] = acc;
    }
    __syncthreads();
    const zc eabc = g.fd[(o + a) * dg] + g.fd[(o + b) * dg] + g.fd[(o + c) * dg];
    zc sum{0.0, 0.0};
    for (int e = threadIdx.x; e < o3; e += NT) {
        const int x = e % o, y = (e / o) % o, z = e / (o * o);
        const zc s1 = Ssh[e];
        const zc wv = s1 + Ssh[z + o * (x + o * y)] + Ssh[y + o * (z + o * x)];
        zc vv = s1;
        for (int q = 0; q < 3; ++q) {
            const int p = trip[q][0], r1 = trip[q][1], r2 = trip[q][2];
            const zc extra = t1[p + (long long)v * x] * g.vvoo[r1 + M * (r2 + (long long)M * (y + (long long)M * z))] +
                             g.fvo[p + (long long)M * x] * t2[r1 + (long long)v * (r2 + (long long)v * (y + (long long)o * z))];
            vv = vv + sgn[q] * extra;
        }
        const zc d = (g.fd[x * dg] + g.fd[y * dg] + g.fd[z * dg]) - eabc;
        sum = sum + divz(wv, d) * conjz(vv);
    }
    red[threadIdx.x] = sum;
    __syncthreads();
    for (int h = NT / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) g.part[w * g.ntri + t] = red[0];
}

// r_w = 1 / x_w
__global__ void recip_kernel(int n, const zc *x, zc *r) {
    const int w = blockIdx.x * NT + threadIdx.x;
    if (w < n) r[w] = divz(zc{1.0, 0.0}, x[w]);
}

// ProjSz1 / ProjSz2VO (SUCCSD_Boson_cmplx/FPUCC_Tools.f90:171-234): zero the entries of a vo (nd = 2) or
// vvoo (nd = 4) tensor whose spins do not conserve Sz.  MO order [occ alpha (noa), occ beta, vir alpha
// (nva), vir beta]; vvoo keeps aaaa, bbbb, abab, abba, baba, baab, i.e. s_a + s_b = s_i + s_j.
__global__ void sz_mask_kernel(int nd, int o, int v, int noa, int nva, long long total, zc *X) {
    for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
        long long r = e;
        const int a = (int)(r % v);
        r /= v;
        bool keep;
        if (nd == 2) {
            const int i = (int)(r % o);
            keep = (a >= nva) == (i >= noa);
        } else {
            const int b = (int)(r % v);
            r /= v;
            const int i = (int)(r % o);
            r /= o;
            const int j = (int)(r % o);
            keep = ((a >= nva) + (b >= nva)) == ((i >= noa) + (j >= noa));
        }
        if (!keep) X[e] = zc{0.0, 0.0};
    }
}

// ---------------------------------------------------------------- chunk context
struct Ctx {
    cudaStream_t st = 0;
    int npts = 1;
    const Arena *ar = nullptr;  // every device buffer of the call: launches are range-checked against them
    zc *pool = nullptr;  // scratch for operands copied into a contiguous order
    size_t cap = 0, used = 0;
    zc *one = nullptr;   // device constant 1
    zc *take(size_t n) {
        n = (n + 1) & ~(size_t)1;
        if (used + n > cap) return nullptr;
        zc *p = pool + used;
        used += n;
        return p;
    }
};

// The elements [lo, hi] (offsets from p) must lie in one buffer of the arena: a launch whose operands
// reach outside their buffers is refused before it runs.
int in_bounds(const Ctx &x, const zc *p, long long lo, long long hi, const char *what) {
    const char *a = reinterpret_cast<const char *>(p + lo), *b = reinterpret_cast<const char *>(p + hi + 1);
    for (const DevBuf &d : x.ar->bufs) {
        const char *s = static_cast<const char *>(d.p);
        if (a >= s && b <= s + d.bytes) return PHF_OK;
    }
    set_error(PHF_ERR_ARG, std::string("pbarhbarolap: operand outside its buffer in ") + what);
    return PHF_ERR_ARG;
}

// range of a view over npts points
int check_tv(const Ctx &x, const TV &t, int npts, const char *what) {
    long long lo = 0, hi = 0;
    for (int d = 0; d < t.nd; ++d) {
        if (t.dim[d] <= 0) return PHF_OK;
        const long long e = (long long)(t.dim[d] - 1) * t.st[d];
        lo += std::min(0LL, e);
        hi += std::max(0LL, e);
    }
    const long long e = (long long)(npts - 1) * t.ps;
    lo += std::min(0LL, e);
    hi += std::max(0LL, e);
    return in_bounds(x, t.p, lo, hi, what);
}

// range of a GEMM operand: rows x cols over nb0 x nb1 batches
int check_view(const Ctx &x, const void *p, long long rows, long long cols, long long rs, long long cs, long long nb0,
               long long bs0, long long nb1, long long bs1, const char *what) {
    const long long ext[4] = {(rows - 1) * rs, (cols - 1) * cs, (nb0 - 1) * bs0, (nb1 - 1) * bs1};
    long long lo = 0, hi = 0;
    for (long long e : ext) {
        lo += std::min(0LL, e);
        hi += std::max(0LL, e);
    }
    return in_bounds(x, static_cast<const zc *>(p), lo, hi, what);
}

int pool_error() {
    set_error(PHF_ERR_OOM, "pbarhbarolap: contraction scratch exhausted");
    return PHF_ERR_OOM;
}

struct Spec {
    std::string a, b, c;
};

Spec parse(const char *spec) {
    std::string s(spec);
    Spec r;
    const size_t arrow = s.find("->");
    std::string lhs = s.substr(0, arrow);
    r.c = s.substr(arrow + 2);
    const size_t comma = lhs.find(',');
    if (comma == std::string::npos) {
        r.a = lhs;
    } else {
        r.a = lhs.substr(0, comma);
        r.b = lhs.substr(comma + 1);
    }
    return r;
}

int letter_pos(const std::string &s, char c) {
    const size_t p = s.find(c);
    return p == std::string::npos ? -1 : (int)p;
}

// C = beta C + alpha op(A) [op(B)] with the input letters mapped onto C's (no summation): permutations,
// outer products, per-point scalings.  npts = 1 for an operation on shared tensors.
int ew(Ctx &x, const char *spec, zc alpha, const TV &A, const TV *B, zc beta, const TV &C, int npts = -1) {
    if (npts < 0) npts = x.npts;
    const Spec sp = parse(spec);
    if ((int)sp.a.size() != A.nd || (int)sp.c.size() != C.nd || (B && (int)sp.b.size() != B->nd)) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: rank mismatch in ") + spec);
        return PHF_ERR_ARG;
    }
    if (C.ps == 0 && npts > 1) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: shared output of a per-point operation ") + spec);
        return PHF_ERR_ARG;
    }
    EwArgs g{};
    g.nd = C.nd;
    for (int d = 0; d < C.nd; ++d) {
        g.dim[d] = C.dim[d];
        g.cs[d] = C.st[d];
        const int pa = letter_pos(sp.a, sp.c[d]);
        g.as[d] = pa < 0 ? 0 : A.st[pa];
        if (pa >= 0 && A.dim[pa] != C.dim[d]) {
            set_error(PHF_ERR_ARG, std::string("pbarhbarolap: dimension mismatch in ") + spec);
            return PHF_ERR_ARG;
        }
        if (B) {
            const int pb = letter_pos(sp.b, sp.c[d]);
            g.bs[d] = pb < 0 ? 0 : B->st[pb];
            if (pb >= 0 && B->dim[pb] != C.dim[d]) {
                set_error(PHF_ERR_ARG, std::string("pbarhbarolap: dimension mismatch in ") + spec);
                return PHF_ERR_ARG;
            }
        }
    }
    for (char ch : sp.a + sp.b)
        if (letter_pos(sp.c, ch) < 0) {
            set_error(PHF_ERR_ARG, std::string("pbarhbarolap: summed letter in elementwise ") + spec);
            return PHF_ERR_ARG;
        }
    g.cps = C.ps;
    g.aps = A.ps;
    g.bps = B ? B->ps : 0;
    g.C = C.p;
    g.A = A.p;
    g.B = B ? B->p : nullptr;
    g.aconj = A.conj;
    g.bconj = B ? B->conj : 0;
    g.alpha = alpha;
    g.beta = beta;
    g.per = numel(C);
    g.total = g.per * npts;
    if (g.total == 0) return PHF_OK;
    PHF_TRY(check_tv(x, C, npts, spec));
    {
        TV a = A;  // A and B over C's index space (letters absent from an input have stride 0)
        a.nd = C.nd;
        for (int d = 0; d < C.nd; ++d) a.dim[d] = C.dim[d], a.st[d] = g.as[d];
        PHF_TRY(check_tv(x, a, npts, spec));
        if (B) {
            TV bb = *B;
            bb.nd = C.nd;
            for (int d = 0; d < C.nd; ++d) bb.dim[d] = C.dim[d], bb.st[d] = g.bs[d];
            PHF_TRY(check_tv(x, bb, npts, spec));
        }
    }
    ew_kernel<<<blocks_for(g.total), NT, 0, x.st>>>(g);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

// copy a view into a contiguous scratch tensor with its letters in the order `order`
int gather(Ctx &x, const std::string &letters, const TV &A, const std::string &order, TV *out, int npts) {
    TV t;
    t.nd = (int)order.size();
    long long s = 1;
    for (int d = 0; d < t.nd; ++d) {
        const int p = letter_pos(letters, order[d]);
        t.dim[d] = A.dim[p];
        t.st[d] = s;
        s *= t.dim[d];
    }
    t.ps = A.ps == 0 ? 0 : s;
    t.p = x.take((size_t)s * (A.ps == 0 ? 1 : npts));
    if (!t.p) return pool_error();
    const std::string spec = letters + "->" + order;
    PHF_TRY(ew(x, spec.c_str(), ONE, A, nullptr, ZERO, t, A.ps == 0 ? 1 : npts));
    *out = t;
    return PHF_OK;
}

// one candidate grouping of a contraction's letters
struct Plan {
    std::string I, J, K, H;  // row, column, summed and batch letters (each ordered)
    bool copyA = false, copyB = false, tempC = false;
    double cost = 0;
};

// stride of a group in a view with letters `ls`; -1 when the group's letters do not form one stride
// (letters absent from the view have stride 0; a group mixing absent and present letters does not merge)
long long group_stride(const TV &t, const std::string &ls, const std::string &grp, int *present) {
    if (grp.empty()) {
        *present = 0;
        return 0;
    }
    int np = 0;
    for (char c : grp) np += letter_pos(ls, c) >= 0;
    *present = np;
    if (np == 0) return 0;
    if (np != (int)grp.size()) return -1;
    long long s0 = t.st[letter_pos(ls, grp[0])];
    long long expect = s0 * t.dim[letter_pos(ls, grp[0])];
    for (size_t k = 1; k < grp.size(); ++k) {
        const int p = letter_pos(ls, grp[k]);
        if (t.st[p] != expect) return -1;
        expect = t.st[p] * t.dim[p];
    }
    return s0;
}

// C = beta C + alpha sum_{summed letters} op(A) op(B), batched over the chunk's points (npts = 1 with the
// point as an explicit letter for sums over points).  Letters: each appears in at least two operands.
int ein(Ctx &x, const char *spec, zc alpha, const TV &A, const TV &B, zc beta, const TV &C, int npts = -1) {
    if (npts < 0) npts = x.npts;
    const Spec sp = parse(spec);
    if ((int)sp.a.size() != A.nd || (int)sp.b.size() != B.nd || (int)sp.c.size() != C.nd) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: rank mismatch in ") + spec);
        return PHF_ERR_ARG;
    }
    if (C.ps == 0 && npts > 1) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: shared output of a per-point contraction ") + spec);
        return PHF_ERR_ARG;
    }
    // letters of size 1 take no part in the grouping
    auto dim_of = [&](char c) -> int {
        int p;
        if ((p = letter_pos(sp.a, c)) >= 0) return A.dim[p];
        if ((p = letter_pos(sp.b, c)) >= 0) return B.dim[p];
        return C.dim[letter_pos(sp.c, c)];
    };
    std::string all;
    for (char c : sp.a + sp.b + sp.c)
        if (all.find(c) == std::string::npos) all += c;
    std::string hard_H, flexA, flexB, K;
    for (char c : all) {
        const bool ia = letter_pos(sp.a, c) >= 0, ib = letter_pos(sp.b, c) >= 0, ic = letter_pos(sp.c, c) >= 0;
        const int d = dim_of(c);
        if ((ia && dim_of(c) != (ia ? A.dim[letter_pos(sp.a, c)] : d)) || (ib && B.dim[letter_pos(sp.b, c)] != d) ||
            (ic && C.dim[letter_pos(sp.c, c)] != d)) {
            set_error(PHF_ERR_ARG, std::string("pbarhbarolap: dimension mismatch in ") + spec);
            return PHF_ERR_ARG;
        }
        if ((int)ia + (int)ib + (int)ic < 2) {
            set_error(PHF_ERR_ARG, std::string("pbarhbarolap: letter in one operand only in ") + spec);
            return PHF_ERR_ARG;
        }
        if (d == 1) continue;
        if (ia && ib && ic) hard_H += c;
        else if (ia && ic) flexA += c;
        else if (ib && ic) flexB += c;
        else K += c;
    }
    auto sort_by = [&](std::string g, const TV &t, const std::string &ls) {
        std::sort(g.begin(), g.end(), [&](char p, char q) {
            const int a = letter_pos(ls, p), b = letter_pos(ls, q);
            const long long sa = a < 0 ? 0 : t.st[a], sb = b < 0 ? 0 : t.st[b];
            return sa < sb || (sa == sb && p < q);
        });
        return g;
    };
    const int nflex = (int)(flexA.size() + flexB.size());
    Plan best;
    best.cost = -1;
    const double copy_w = 27.0;  // one copied element costs about as much as 27 complex MACs
    for (int mask = 0; mask < (1 << nflex); ++mask) {
        for (int kord = 0; kord < 2; ++kord) {
            Plan p;
            std::string H = hard_H, I, J;
            for (int q = 0; q < nflex; ++q) {
                const char c = q < (int)flexA.size() ? flexA[q] : flexB[q - flexA.size()];
                if (mask >> q & 1) H += c;
                else if (q < (int)flexA.size()) I += c;
                else J += c;
            }
            p.I = sort_by(I, C, sp.c);
            p.J = sort_by(J, C, sp.c);
            p.H = sort_by(H, C, sp.c);
            p.K = kord == 0 ? sort_by(K, A, sp.a) : sort_by(K, B, sp.b);
            int pr;
            // C must hold I, J, H each as one stride
            p.tempC = group_stride(C, sp.c, p.I, &pr) < 0 || group_stride(C, sp.c, p.J, &pr) < 0 ||
                      group_stride(C, sp.c, p.H, &pr) < 0;
            p.copyA = group_stride(A, sp.a, p.I, &pr) < 0 || group_stride(A, sp.a, p.K, &pr) < 0 ||
                      group_stride(A, sp.a, p.H, &pr) < 0;
            p.copyB = group_stride(B, sp.b, p.K, &pr) < 0 || group_stride(B, sp.b, p.J, &pr) < 0 ||
                      group_stride(B, sp.b, p.H, &pr) < 0;
            // a batch group mixing letters present and absent in an operand stays unmergeable after a copy
            int ha, hb;
            group_stride(A, sp.a, p.H, &ha);
            group_stride(B, sp.b, p.H, &hb);
            if ((ha != 0 && ha != (int)p.H.size()) || (hb != 0 && hb != (int)p.H.size())) continue;
            double m = 1, n = 1, k = 1, nb = 1;
            for (char c : p.I) m *= dim_of(c);
            for (char c : p.J) n *= dim_of(c);
            for (char c : p.K) k *= dim_of(c);
            for (char c : p.H) nb *= dim_of(c);
            const double pts = (A.ps == 0 && B.ps == 0) ? 1 : npts;
            // tile 64 x 64 padding (the narrow tiles help only some shapes), per-CTA overhead of ~2 k-steps
            p.cost = pts * nb * std::ceil(m / 64) * 64 * std::ceil(n / 64) * 64 * (k + 32);
            if (p.copyA) p.cost += copy_w * (A.ps == 0 ? 1 : npts) * (double)numel(A);
            if (p.copyB) p.cost += copy_w * (B.ps == 0 ? 1 : npts) * (double)numel(B);
            if (p.tempC) p.cost += 2 * copy_w * npts * (double)numel(C);
            if (best.cost < 0 || p.cost < best.cost) best = p;
        }
    }
    if (best.cost < 0) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: no GEMM grouping for ") + spec);
        return PHF_ERR_ARG;
    }
    const size_t mark = x.used;
    TV a = A, b = B;
    std::string la = sp.a, lb = sp.b;
    if (best.copyA) {
        std::string order = best.I + best.K;
        for (char c : best.H)
            if (letter_pos(sp.a, c) >= 0) order += c;
        for (char c : sp.a)
            if (order.find(c) == std::string::npos) order += c;  // size-1 letters
        PHF_TRY(gather(x, sp.a, A, order, &a, npts));
        la = order;
    }
    if (best.copyB) {
        std::string order = best.K + best.J;
        for (char c : best.H)
            if (letter_pos(sp.b, c) >= 0) order += c;
        for (char c : sp.b)
            if (order.find(c) == std::string::npos) order += c;
        PHF_TRY(gather(x, sp.b, B, order, &b, npts));
        lb = order;
    }
    TV c = C;
    std::string lc = sp.c;
    if (best.tempC) {
        std::string order = best.I + best.J + best.H;
        for (char ch : sp.c)
            if (order.find(ch) == std::string::npos) order += ch;
        TV t;
        t.nd = (int)order.size();
        long long s = 1;
        for (int d = 0; d < t.nd; ++d) {
            t.dim[d] = C.dim[letter_pos(sp.c, order[d])];
            t.st[d] = s;
            s *= t.dim[d];
        }
        t.ps = C.ps == 0 ? 0 : s;
        t.p = x.take((size_t)s * (C.ps == 0 ? 1 : npts));
        if (!t.p) return pool_error();
        c = t;
        lc = order;
    }
    int pr;
    long long m = 1, n = 1, k = 1, nb = 1;
    for (char ch : best.I) m *= dim_of(ch);
    for (char ch : best.J) n *= dim_of(ch);
    for (char ch : best.K) k *= dim_of(ch);
    for (char ch : best.H) nb *= dim_of(ch);
    View va, vb;
    va.p = a.p;
    va.rs = group_stride(a, la, best.I, &pr);
    va.cs = group_stride(a, la, best.K, &pr);
    va.bs0 = a.ps;
    va.bs1 = group_stride(a, la, best.H, &pr);
    va.conj = a.conj;
    vb.p = b.p;
    vb.rs = group_stride(b, lb, best.K, &pr);
    vb.cs = group_stride(b, lb, best.J, &pr);
    vb.bs0 = b.ps;
    vb.bs1 = group_stride(b, lb, best.H, &pr);
    vb.conj = b.conj;
    OutView vc;
    vc.p = c.p;
    vc.rs = group_stride(c, lc, best.I, &pr);
    vc.cs = group_stride(c, lc, best.J, &pr);
    vc.bs0 = c.ps;
    vc.bs1 = group_stride(c, lc, best.H, &pr);
    if (va.rs < 0 || va.cs < 0 || va.bs1 < 0 || vb.rs < 0 || vb.cs < 0 || vb.bs1 < 0 || vc.rs < 0 || vc.cs < 0 ||
        vc.bs1 < 0) {
        set_error(PHF_ERR_ARG, std::string("pbarhbarolap: internal grouping error in ") + spec);
        return PHF_ERR_ARG;
    }
    if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || nb > INT32_MAX) {
        set_error(PHF_ERR_UNSUPPORTED, std::string("pbarhbarolap: contraction too large: ") + spec);
        return PHF_ERR_UNSUPPORTED;
    }
    const int pts = (A.ps == 0 && B.ps == 0 && C.ps == 0) ? 1 : npts;
    PHF_TRY(check_view(x, va.p, m, k, va.rs, va.cs, pts, va.bs0, nb, va.bs1, spec));
    PHF_TRY(check_view(x, vb.p, k, n, vb.rs, vb.cs, pts, vb.bs0, nb, vb.bs1, spec));
    PHF_TRY(check_view(x, vc.p, m, n, vc.rs, vc.cs, pts, vc.bs0, nb, vc.bs1, spec));
    const zc cbeta = best.tempC ? ZERO : beta;
    const long long tiles = (long long)pts * nb * ((m + 63) / 64) * ((n + 63) / 64);
    if (m == 1 && n == 1 && nb == 1 && k >= 256) {
        // a scalar per point: a blocked dot product, k split over S CTAs per point, then the sum of the parts
        const int S = (int)std::max<long long>(1, std::min<long long>(k / 2048 + 1, (8 * 148 + pts - 1) / pts));
        zc *T = x.take((size_t)S * pts);
        if (!T) return pool_error();
        PHF_TRY(check_view(x, T, 1, 1, 0, 0, pts, S, S, 1, spec));
        dot_kernel<<<(unsigned)(pts * S), NT, 0, x.st>>>(k, S, va, vb, T);
        ++g_launches;
        PHF_CHECK_LAUNCH();
        splitk_reduce_kernel<<<blocks_for(pts), NT, 0, x.st>>>(1, 1, S, pts, T, vc, alpha, cbeta);
        ++g_launches;
        PHF_CHECK_LAUNCH();
    } else if (nb == 1 && tiles < 2 * 148 && k >= 1024) {
        // few output tiles and a long k: split k over S batches of partial products, then sum them
        const int S = (int)std::max<long long>(2, std::min<long long>(k / 256, (4 * 148 + tiles - 1) / tiles));
        const long long ks = k / S, rem = k - S * ks;
        zc *T = x.take((size_t)(m * n * S) * pts);
        if (!T) return pool_error();
        View a2 = va, b2 = vb;
        a2.bs1 = ks * va.cs;
        b2.bs1 = ks * vb.rs;
        OutView t2;
        t2.p = T;
        t2.rs = 1;
        t2.cs = m;
        t2.bs0 = m * n * S;
        t2.bs1 = m * n;
        PHF_TRY(check_view(x, T, m, n, 1, m, pts, m * n * S, S, m * n, spec));
        PHF_TRY(zgemm_strided((int)m, (int)n, (int)ks, pts, S, ONE, a2, b2, ZERO, t2, nullptr, x.st));
        if (rem) {
            View a3 = va, b3 = vb;
            a3.p = static_cast<const zc *>(va.p) + S * ks * va.cs;
            b3.p = static_cast<const zc *>(vb.p) + S * ks * vb.rs;
            OutView t3 = t2;
            t3.bs1 = 0;
            PHF_TRY(zgemm_strided((int)m, (int)n, (int)rem, pts, 1, ONE, a3, b3, ONE, t3, nullptr, x.st));
        }
        const long long total = m * n * pts;
        splitk_reduce_kernel<<<blocks_for(total), NT, 0, x.st>>>((int)m, (int)n, S, total, T, vc, alpha, cbeta);
        ++g_launches;
        PHF_CHECK_LAUNCH();
    } else {
        PHF_TRY(zgemm_strided((int)m, (int)n, (int)k, pts, (int)nb, alpha, va, vb, cbeta, vc, nullptr, x.st));
    }
    g_pcc_flops += 8.0 * (double)m * (double)n * (double)k * (double)nb * pts;
    if (best.tempC) {
        const std::string back = lc + "->" + sp.c;
        PHF_TRY(ew(x, back.c_str(), ONE, c, nullptr, beta, C, pts));
    }
    x.used = mark;
    return PHF_OK;
}

int mask_sz(Ctx &x, const TV &t, int o, int v, int nao) {
    const int noa = o / 2, nva = nao - noa;
    const long long total = numel(t) * x.npts;
    if (t.ps != numel(t) && x.npts > 1) {
        set_error(PHF_ERR_ARG, "pbarhbarolap: ProjSz on a non-contiguous tensor");
        return PHF_ERR_ARG;
    }
    PHF_TRY(in_bounds(x, t.p, 0, total - 1, "ProjSz"));
    sz_mask_kernel<<<blocks_for(total), NT, 0, x.st>>>(t.nd, o, v, noa, nva, total, t.p);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

// Wigner (SUCCSD_Boson_cmplx/Wrappers.f90:769-797), arguments in its declared order (J, N, M):
// exp(-i N alpha) d^J_{NM}(beta) exp(-i M gama)
cd wigner_pcc(int j, int n, int m, double alpha, double beta, double gama) {
    double fac = std::sqrt(std::tgamma(j + n + 1.0) * std::tgamma(j - n + 1.0) * std::tgamma(j + m + 1.0) *
                           std::tgamma(j - m + 1.0));
    double d = 0.0;
    for (int s = std::max(0, m - n); s <= std::min(j + m, j - n); ++s) {
        const int p1 = n - m + s, p2 = 2 * j + m - n - 2 * s, p3 = n - m + 2 * s;
        const double numer = ((p1 & 1) ? -1.0 : 1.0) * std::pow(std::cos(beta / 2), p2) * std::pow(std::sin(beta / 2), p3);
        d += numer / (std::tgamma(j + m - s + 1.0) * std::tgamma(s + 1.0) * std::tgamma(n - m + s + 1.0) *
                      std::tgamma(j - n - s + 1.0));
    }
    return std::exp(cd(0.0, -n * alpha)) * (d * fac) * std::exp(cd(0.0, -m * gama));
}

}  // namespace

// PbarHbarOlap (SUCCSD_Boson_cmplx/FPUCC.f90:14-272).  Host arrays in the reference's Fortran layouts.
int pbarhbarolap_run(const PccArgs &g, phf_complex *olap0, phf_complex *olapex1, phf_complex *olapex2,
                     phf_complex *eolap0, phf_complex *eolapex1, phf_complex *eolapex2) {
    const int M = g.nso, o = g.nocc, v = M - o, nl = g.npoints[0], ny = g.npoints[1], npg = g.npg;
    const int nao = M / 2;
    const long long M2 = (long long)M * M, M4 = M2 * M2, vo = (long long)v * o, vvoo = vo * vo;
    const long long v4 = (long long)v * v * v * v, o4 = (long long)o * o * o * o;
    const int nw = nl * ny * npg;
    const bool sz = g.sp == 2;

    // per-point weight: sum over the Wigner pairs (m, n) and point-group components (p, q)  (:160-176)
    std::vector<cd> wt(nw);
    for (int ia = 0; ia < nl; ++ia)
        for (int iy = 0; iy < ny; ++iy)
            for (int ig = 0; ig < npg; ++ig) {
                cd acc = 0;
                for (int mm = -g.qj; mm <= g.qj; ++mm)
                    for (int nn = -g.qj; nn <= g.qj; ++nn)
                        for (int p = 0; p < g.ncipg; ++p)
                            for (int q = 0; q < g.ncipg; ++q) {
                                const cd wig = g.sp == 2 ? wigner_pcc(g.qj, mm, nn, g.roota[ia], g.rootb[iy], g.rooty[ia])
                                                         : wigner_pcc(g.qj, mm, nn, g.roota[ia], g.rootb[ia], g.rooty[iy]);
                                cd w = g.weightsp[(size_t)ia + (size_t)nl * iy] *
                                       g.weightpg[(size_t)ig + (size_t)npg * ((size_t)p + (size_t)g.ncipg * q)];
                                w = wig * w * std::conj(cd(g.fsp[g.qj + mm].re, g.fsp[g.qj + mm].im)) *
                                    cd(g.fsp[g.qj + nn].re, g.fsp[g.qj + nn].im);
                                acc += w * std::conj(cd(g.fpg[p].re, g.fpg[p].im)) * cd(g.fpg[q].re, g.fpg[q].im);
                            }
                wt[((size_t)ia * ny + iy) * npg + ig] = acc;
            }

    // chunk size from the workspace budget
    const size_t per = (size_t)(3 * M4 + 2 * (long long)v * v * o * M + (long long)v * v * M2 + (long long)v * M * M2 +
                                v4 + 2 * (long long)o * o * v * v + o4 + (long long)o * o * o * v + 18 * vvoo +
                                8 * M2 + 12 * vo + 4 * (long long)v * v + 4 * (long long)o * o + 32) *
                       sizeof(zc);
    const size_t budget = g.workspace ? g.workspace : ((size_t)16 << 30);
    const int b = (int)std::max<size_t>(1, std::min<size_t>(budget / per, (size_t)nw));

    Arena ar;
    zc *H1 = nullptr, *H2 = nullptr, *T1 = nullptr, *T2 = nullptr, *R1 = nullptr, *R2 = nullptr, *Rpg = nullptr,
       *Rk2 = nullptr, *wtd = nullptr, *one = nullptr;
    long long *offs = nullptr;
    auto up = [&](const phf_complex *src, long long n, zc **dst) -> int {
        PHF_TRY(ar.alloc(dst, (size_t)n));
        PHF_CUDA(cudaMemcpy(*dst, src, (size_t)n * sizeof(zc), cudaMemcpyHostToDevice));
        return PHF_OK;
    };
    // rotations column-major per index: R(i, j) of entry t at t M^2 + i + M j
    auto rot = [&](const phf_complex *src, int cnt, int first, int take, zc **dst) -> int {
        PHF_TRY(ar.alloc(dst, (size_t)take * M2));
        std::vector<zc> h((size_t)take * M2);
        for (int t = 0; t < take; ++t)
            for (int j = 0; j < M; ++j)
                for (int i = 0; i < M; ++i) {
                    const phf_complex e = src[(size_t)(first + t) + (size_t)cnt * ((size_t)i + (size_t)M * j)];
                    h[(size_t)t * M2 + i + (size_t)M * j] = zc{e.re, e.im};
                }
        PHF_CUDA(cudaMemcpy(*dst, h.data(), h.size() * sizeof(zc), cudaMemcpyHostToDevice));
        return PHF_OK;
    };
    PHF_TRY(up(g.hone, M2, &H1));
    PHF_TRY(up(g.htwo, M4, &H2));
    PHF_TRY(up(g.t1, vo, &T1));
    PHF_TRY(up(g.t2, vvoo, &T2));
    PHF_TRY(rot(g.r1, nl, 0, nl, &R1));
    PHF_TRY(rot(g.r2, ny, 0, ny, &R2));
    PHF_TRY(rot(g.rpg, npg, 0, npg, &Rpg));
    if (g.ncik == 2) PHF_TRY(rot(g.rk, g.ncik, 1, 1, &Rk2));
    PHF_TRY(ar.alloc(&wtd, (size_t)nw));
    PHF_CUDA(cudaMemcpy(wtd, wt.data(), nw * sizeof(zc), cudaMemcpyHostToDevice));
    PHF_TRY(ar.alloc(&one, 1));
    PHF_CUDA(cudaMemcpy(one, &ONE, sizeof(zc), cudaMemcpyHostToDevice));
    // GEMM offsets: T_w = R2[iy] Rpg[ipg], then R_w = R1[il] T_w
    {
        std::vector<long long> o1(6 * (size_t)nw);
        for (int w = 0; w < nw; ++w) {
            const int il = w / (ny * npg), iy = (w / npg) % ny, ig = w % npg;
            o1[3 * w] = (long long)iy * M2;
            o1[3 * w + 1] = (long long)ig * M2;
            o1[3 * w + 2] = 0;
            o1[3 * (size_t)nw + 3 * w] = (long long)il * M2;
            o1[3 * (size_t)nw + 3 * w + 1] = 0;
            o1[3 * (size_t)nw + 3 * w + 2] = 0;
        }
        PHF_TRY(ar.alloc(&offs, 6 * (size_t)nw));
        PHF_CUDA(cudaMemcpy(offs, o1.data(), o1.size() * sizeof(long long), cudaMemcpyHostToDevice));
    }

    // shared: Fock matrix and E_SCF of the pass's Hamiltonian, conjugated copies for the ncik = 2 pass
    zc *F = nullptr, *escf = nullptr, *H1c = nullptr, *H2c = nullptr, *T1c = nullptr, *T2c = nullptr;
    PHF_TRY(ar.alloc(&F, (size_t)M2));
    PHF_TRY(ar.alloc(&escf, 1));
    if (g.ncik == 2) {
        PHF_TRY(ar.alloc(&H1c, (size_t)M2));
        PHF_TRY(ar.alloc(&H2c, (size_t)M4));
        PHF_TRY(ar.alloc(&T1c, (size_t)vo));
        PHF_TRY(ar.alloc(&T2c, (size_t)vvoo));
    }
    // chunk workspace
    auto A = [&](zc **p, long long n) { return ar.alloc(p, (size_t)b * (size_t)n); };
    zc *R = nullptr, *Tm = nullptr, *Y0 = nullptr, *Linv = nullptr, *U0 = nullptr, *U1 = nullptr, *V = nullptr,
       *Vinv = nullptr, *Ut = nullptr, *X1 = nullptr, *X2 = nullptr, *X3 = nullptr, *Fw = nullptr, *E0 = nullptr,
       *C0 = nullptr, *C1 = nullptr, *C2 = nullptr, *rC0 = nullptr, *W0 = nullptr, *W1 = nullptr, *W2 = nullptr,
       *tmp = nullptr, *det2 = nullptr, *ldet = nullptr;
    zc *itm1 = nullptr, *tau = nullptr, *tb = nullptr, *itm4 = nullptr, *Fvv = nullptr, *Foo = nullptr, *Fov = nullptr,
       *Wo = nullptr, *Wv = nullptr, *Wovvo = nullptr, *itm4b = nullptr, *itm2 = nullptr, *r1 = nullptr, *res2 = nullptr,
       *itm1p = nullptr, *itm3p = nullptr, *Ovl2 = nullptr, *EO0 = nullptr, *EO1 = nullptr, *EO2 = nullptr,
       *sw = nullptr;
    int *flag = nullptr;
    PHF_TRY(A(&R, M2));
    PHF_TRY(A(&Tm, M2));
    PHF_TRY(A(&Y0, (long long)M * o));
    PHF_TRY(A(&Linv, (long long)o * o));
    PHF_TRY(A(&U0, 1));
    PHF_TRY(A(&U1, vo));
    PHF_TRY(A(&V, M2));
    PHF_TRY(A(&Vinv, M2));
    PHF_TRY(A(&Ut, M4));
    PHF_TRY(A(&X1, (long long)v * v * o * M));
    PHF_TRY(A(&X2, (long long)v * v * M2));
    PHF_TRY(A(&X3, (long long)v * M * M2));
    PHF_TRY(A(&Fw, M2));
    PHF_TRY(A(&E0, 1));
    PHF_TRY(A(&C0, 1));
    PHF_TRY(A(&C1, vo));
    PHF_TRY(A(&C2, vvoo));
    PHF_TRY(A(&rC0, 1));
    PHF_TRY(A(&W0, 1));
    PHF_TRY(A(&W1, vo));
    PHF_TRY(A(&W2, vvoo));
    PHF_TRY(A(&tmp, vvoo));
    PHF_TRY(A(&det2, 1));
    PHF_TRY(A(&ldet, 1));
    PHF_TRY(A(&itm1, vvoo));
    PHF_TRY(A(&tau, vvoo));
    PHF_TRY(A(&tb, vvoo));
    PHF_TRY(A(&itm4, vvoo));
    PHF_TRY(A(&Fvv, (long long)v * v));
    PHF_TRY(A(&Foo, (long long)o * o));
    PHF_TRY(A(&Fov, vo));
    PHF_TRY(A(&Wo, o4));
    PHF_TRY(A(&Wv, v4));
    PHF_TRY(A(&Wovvo, vvoo));
    PHF_TRY(A(&itm4b, (long long)o * o * o * v));
    PHF_TRY(A(&itm2, vvoo));
    PHF_TRY(A(&r1, vo));
    PHF_TRY(A(&res2, vvoo));
    PHF_TRY(A(&itm1p, (long long)v * v));
    PHF_TRY(A(&itm3p, (long long)o * o));
    PHF_TRY(A(&Ovl2, vvoo));
    PHF_TRY(A(&EO0, 1));
    PHF_TRY(A(&EO1, vo));
    PHF_TRY(A(&EO2, vvoo));
    PHF_TRY(A(&sw, 1));
    PHF_TRY(ar.alloc(&flag, 1));
    Ctx x;
    x.ar = &ar;
    x.one = one;
    // (T) energy (TrunODE 3): the W tensor of a few points at a time, the triples a >= b >= c
    const long long o3v3 = (long long)o * o * o * v * v * v;
    x.cap = (size_t)b * (size_t)(2 * M4 + 64);
    PHF_TRY(ar.alloc(&x.pool, x.cap));
    const long long ntri = (long long)v * (v + 1) * (v + 2) / 6;
    int nsubT = 0;
    zc *Wtrip = nullptr, *tpart = nullptr;
    int *trid = nullptr;
    // the W tensor of a point with its GEMM operands (rows (x,b,c) x k = v + o, k x columns (a,y,z))
    const long long tens_per = o3v3 + ((long long)o * v * v + (long long)v * o * o) * (v + o);
    const long long by_budget = (long long)(budget / 2) / (tens_per * (long long)sizeof(zc));
    // W per point in half the workspace: the GEMM path; else, for o <= 18, one o^3 sum per triple in
    // shared memory
    const bool fusedT = by_budget < 1 && o <= kTriplesFusedMaxO;
    zc *Aop = nullptr, *Bop = nullptr;
    if (g.trunode == 3) {
        if (by_budget < 1 && !fusedT) {
            set_error(PHF_ERR_UNSUPPORTED, "pbarhbarolap: the (T) tensor of one point exceeds the workspace");
            return PHF_ERR_UNSUPPORTED;
        }
        nsubT = fusedT ? b : (int)std::min<long long>((long long)b, by_budget);
        if (!fusedT) {
            PHF_TRY(ar.alloc(&Wtrip, (size_t)nsubT * (size_t)o3v3));
            PHF_TRY(ar.alloc(&Aop, (size_t)nsubT * (size_t)((long long)o * v * v * (v + o))));
            PHF_TRY(ar.alloc(&Bop, (size_t)nsubT * (size_t)((long long)v * o * o * (v + o))));
        }
        PHF_TRY(ar.alloc(&tpart, (size_t)nsubT * (size_t)ntri));
        PHF_TRY(ar.alloc(&trid, 3 * (size_t)ntri));
        std::vector<int> tr;
        tr.reserve(3 * (size_t)ntri);
        for (int a = 0; a < v; ++a)      // the order of the reference's loops (CCSD_T.f90:38-40)
            for (int bb = 0; bb <= a; ++bb)
                for (int c = 0; c <= bb; ++c) tr.insert(tr.end(), {a, bb, c});
        PHF_CUDA(cudaMemcpy(trid, tr.data(), tr.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // accumulators: eps0, lambda0, eps1, lambda1, eps2, lambda2
    zc *acc = nullptr;
    const long long nacc = 2 + 2 * vo + 2 * vvoo;
    PHF_TRY(ar.alloc(&acc, (size_t)nacc));
    zc *aE0 = acc, *aL0 = acc + 1, *aE1 = acc + 2, *aL1 = aE1 + vo, *aE2 = aL1 + vo, *aL2 = aE2 + vvoo;
    const cudaStream_t st = x.st;
    PHF_CUDA(cudaMemsetAsync(acc, 0, nacc * sizeof(zc), st));
    PHF_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));

    // views shared by all points
    auto sh = [](TV t) {
        t.ps = 0;
        return t;
    };
    const TV ones1 = [&] {
        TV t = scal(one, false);
        return t;
    }();
    auto ones_v = [&](int d0, int d1 = 0) {  // all-ones tensor of one or two indices (strides 0)
        TV t;
        t.p = one;
        t.nd = d1 ? 2 : 1;
        t.dim[0] = d0;
        t.dim[1] = d1;
        return t;
    };

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    PHF_CUDA(cudaEventCreate(&ev0));
    PHF_CUDA(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{ev0, ev1};
    g_pcc_flops = 0.0;
    PHF_CUDA(cudaEventRecord(ev0, st));
    for (int pass = 0; pass < (g.ncik == 2 ? 2 : 1); ++pass) {
        const zc *h1 = pass ? H1c : H1;
        zc *h2 = pass ? H2c : H2;
        zc *t1 = pass ? T1c : T1;
        zc *t2 = pass ? T2c : T2;
        x.npts = 1;
        if (pass) {  // EvalKernel(Conjg(HOne), Conjg(HTwo), Conjg(T1), Conjg(T2), ...) (:194-197)
            PHF_TRY(ew(x, "pq->pq", ONE, conjv(tens(H1, {M, M}, false)), nullptr, ZERO, tens(H1c, {M, M}, false), 1));
            PHF_TRY(ew(x, "pqrs->pqrs", ONE, conjv(tens(H2, {M, M, M, M}, false)), nullptr, ZERO,
                       tens(H2c, {M, M, M, M}, false), 1));
            PHF_TRY(ew(x, "ai->ai", ONE, conjv(tens(T1, {v, o}, false)), nullptr, ZERO, tens(T1c, {v, o}, false), 1));
            PHF_TRY(ew(x, "abij->abij", ONE, conjv(tens(T2, {v, v, o, o}, false)), nullptr, ZERO,
                       tens(T2c, {v, v, o, o}, false), 1));
        }
        const TV H2v = tens(h2, {M, M, M, M}, false);
        const TV Fv = tens(F, {M, M}, false);
        // MKFock_MO (UHF.f90:461-500): F = h + sum_i <p i||q i>, E_SCF = sum_i h_ii + sum_ij <ij||ij>/2, + ENuc
        {
            PHF_TRY(ew(x, "pq->pq", ONE, tens(const_cast<zc *>(h1), {M, M}, false), nullptr, ZERO, Fv, 1));
            TV dg;  // H2(p, i, q, i)
            dg.p = h2;
            dg.nd = 3;
            dg.dim[0] = M, dg.dim[1] = o, dg.dim[2] = M;
            dg.st[0] = 1, dg.st[1] = M + M * M2, dg.st[2] = M2;
            PHF_TRY(ein(x, "piq,i->pq", ONE, dg, ones_v(o), ONE, Fv, 1));
            TV hd;  // h(i, i)
            hd.p = const_cast<zc *>(h1);
            hd.nd = 1;
            hd.dim[0] = o;
            hd.st[0] = M + 1;
            const zc en{g.enuc, 0.0};
            PHF_TRY(ew(x, "->", en, ones1, nullptr, ZERO, scal(escf, false), 1));
            PHF_TRY(ein(x, "i,i->", ONE, hd, ones_v(o), ONE, scal(escf, false), 1));
            TV d2;  // H2(i, j, i, j)
            d2.p = h2;
            d2.nd = 2;
            d2.dim[0] = o, d2.dim[1] = o;
            d2.st[0] = 1 + M2, d2.st[1] = M + M * M2;
            PHF_TRY(ein(x, "ij,ij->", mkz(0.5), d2, ones_v(o, o), ONE, scal(escf, false), 1));
        }
        const TV T1s = tens(t1, {v, o}, false), T2s = tens(t2, {v, v, o, o}, false);
        const TV Hoovv = blk(H2v, {0, 0, o, o}, {o, o, v, v}), Hooov = blk(H2v, {0, 0, 0, o}, {o, o, o, v}),
                 Hoovo = blk(H2v, {0, 0, o, 0}, {o, o, v, o}), Hvovv = blk(H2v, {o, 0, o, o}, {v, o, v, v}),
                 Hovvv = blk(H2v, {0, o, o, o}, {o, v, v, v}), Hvoov = blk(H2v, {o, 0, 0, o}, {v, o, o, v}),
                 Hovvo = blk(H2v, {0, o, o, 0}, {o, v, v, o}), Hvvoo = blk(H2v, {o, o, 0, 0}, {v, v, o, o}),
                 Hvvvo = blk(H2v, {o, o, o, 0}, {v, v, v, o}), Hovoo = blk(H2v, {0, o, 0, 0}, {o, v, o, o}),
                 Hoooo = blk(H2v, {0, 0, 0, 0}, {o, o, o, o}), Hvvvv = blk(H2v, {o, o, o, o}, {v, v, v, v});
        const TV Fov_s = blk(Fv, {0, o}, {o, v}), Fvo_s = blk(Fv, {o, 0}, {v, o}), Foo_s = blk(Fv, {0, 0}, {o, o}),
                 Fvv_s = blk(Fv, {o, o}, {v, v});

        for (int w0 = 0; w0 < nw; w0 += b) {
            const int bc = std::min(b, nw - w0);
            x.npts = bc;
            x.used = 0;
            const TV Rv = tens(R, {M, M}), Y0v = tens(Y0, {M, o}), U1v = tens(U1, {v, o}), Vv = tens(V, {M, M}),
                     Viv = tens(Vinv, {M, M}), Utv = tens(Ut, {M, M, M, M}), Fwv = tens(Fw, {M, M});
            // fixed-shape launches of this chunk: operands within their buffers
            PHF_TRY(check_view(x, Tm, M, M, 1, M, bc, M2, 1, 0, "R products"));
            PHF_TRY(check_view(x, R, M, M, 1, M, bc, M2, 1, 0, "R products"));
            PHF_TRY(check_view(x, V, M, M, 1, M, bc, M2, 1, 0, "V"));
            PHF_TRY(check_view(x, Vinv, M, M, 1, M, bc, M2, 1, 0, "V inverse"));
            PHF_TRY(check_view(x, Y0, o, o, M, 1, bc, (long long)M * o, 1, 0, "occupied block"));
            PHF_TRY(check_view(x, Linv, o, o, o, 1, bc, (long long)o * o, 1, 0, "occupied inverse"));
            PHF_TRY(check_view(x, C0, 1, 1, 0, 0, bc, 1, 1, 0, "C0"));
            PHF_TRY(check_view(x, rC0, 1, 1, 0, 0, bc, 1, 1, 0, "1/C0"));
            PHF_TRY(check_view(x, U0, 1, 1, 0, 0, bc, 1, 1, 0, "det"));
            PHF_TRY(check_view(x, det2, 1, 1, 0, 0, bc, 1, 1, 0, "det"));
            PHF_TRY(check_view(x, ldet, 1, 1, 0, 0, bc, 1, 1, 0, "logdet"));
            PHF_TRY(check_view(x, R2, M, M, 1, M, ny, M2, 1, 0, "R2"));
            PHF_TRY(check_view(x, Rpg, M, M, 1, M, npg, M2, 1, 0, "Rpg"));
            PHF_TRY(check_view(x, R1, M, M, 1, M, nl, M2, 1, 0, "R1"));
            // R_w = R1[il] (R2[iy] Rpg[ipg]) [Rk(2)]  (:189-192)
            PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, View{R2, 1, M}, View{Rpg, 1, M}, ZERO,
                                  OutView{Tm, 1, M, M2}, offs + 3LL * w0, st));
            if (pass) {
                PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, View{R1, 1, M}, View{Tm, 1, M, M2}, ZERO,
                                      OutView{V, 1, M, M2}, offs + 3LL * nw + 3LL * w0, st));
                PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, View{V, 1, M, M2}, View{Rk2, 1, M}, ZERO,
                                      OutView{R, 1, M, M2}, nullptr, st));
            } else {
                PHF_TRY(zgemm_strided(M, M, M, bc, 1, ONE, View{R1, 1, M}, View{Tm, 1, M, M2}, ZERO,
                                      OutView{R, 1, M, M2}, offs + 3LL * nw + 3LL * w0, st));
            }
            // ProjT1: Y0 = R [1; T1] (first o columns), U0 = det Y0[:o], U1 = Y0[o:] Y0[:o]^-1
            PHF_TRY(ew(x, "pi->pi", ONE, blk(Rv, {0, 0}, {M, o}), nullptr, ZERO, Y0v));
            PHF_TRY(ein(x, "pa,ai->pi", ONE, blk(Rv, {0, o}, {M, v}), T1s, ONE, Y0v));
            // column-major blocks read as row-major give the transposed matrix; its row-major inverse is the
            // column-major inverse, and the determinant is the same
            PHF_TRY(overlap_inverse(o, bc, Y0, M, (long long)M * o, Linv, o, (long long)o * o, U0, ldet, flag, st));
            PHF_TRY(ein(x, "ak,ki->ai", ONE, blk(Y0v, {o, 0}, {v, o}), tens(Linv, {o, o}), ZERO, U1v));
            // TransT2 with T1 = U1: V = [1 0; -U1 1] R (PCCCI.f90:139-142), V^-1
            PHF_TRY(ew(x, "pq->pq", ONE, Rv, nullptr, ZERO, Vv));
            PHF_TRY(ein(x, "ai,iq->aq", mkz(-1), U1v, blk(Rv, {0, 0}, {o, M}), ONE, blk(Vv, {o, 0}, {v, M})));
            PHF_TRY(overlap_inverse(M, bc, V, M, M2, Vinv, M, M2, det2, ldet, flag, st));
            // U'(p,q,r,s) = sum V(p,a) V(q,b) T2(a,b,c,d) V^-1(c,r) V^-1(d,s) over a, b virtual, c, d occupied
            // (IntTran4Sim of the T2-only tensor, IntTrans.f90:486-572)
            const TV X1v = tens(X1, {v, v, o, M}), X2v = tens(X2, {v, v, M, M}), X3v = tens(X3, {v, M, M, M});
            PHF_TRY(ein(x, "abcd,ds->abcs", ONE, T2s, blk(Viv, {0, 0}, {o, M}), ZERO, X1v));
            PHF_TRY(ein(x, "abcs,cr->abrs", ONE, X1v, blk(Viv, {0, 0}, {o, M}), ZERO, X2v));
            PHF_TRY(ein(x, "abrs,qb->aqrs", ONE, X2v, blk(Vv, {0, o}, {M, v}), ZERO, X3v));
            PHF_TRY(ein(x, "pa,aqrs->pqrs", ONE, blk(Vv, {0, o}, {M, v}), X3v, ZERO, Utv));
            // MKFock_MO(0, U'): F_w(p,q) = sum_i U'(p,i,q,i), E0 = sum_ij U'(i,j,i,j)/2  (PCCCI.f90:146)
            {
                TV dg = Utv;
                dg.nd = 3;
                dg.dim[0] = M, dg.dim[1] = o, dg.dim[2] = M;
                dg.st[0] = 1, dg.st[1] = M + M * M2, dg.st[2] = M2;
                PHF_TRY(ein(x, "piq,i->pq", ONE, dg, ones_v(o), ZERO, Fwv));
                TV d2 = Utv;
                d2.nd = 2;
                d2.dim[0] = o, d2.dim[1] = o;
                d2.st[0] = 1 + M2, d2.st[1] = M + M * M2;
                PHF_TRY(ein(x, "ij,ij->", mkz(0.5), d2, ones_v(o, o), ZERO, scal(E0)));
            }
            const TV fov = blk(Fwv, {0, o}, {o, v}), fvo = blk(Fwv, {o, 0}, {v, o}), foo = blk(Fwv, {0, 0}, {o, o}),
                     fvv = blk(Fwv, {o, o}, {v, v});
            const TV uvvoo = blk(Utv, {o, o, 0, 0}, {v, v, o, o}), uoovv = blk(Utv, {0, 0, o, o}, {o, o, v, v}),
                     uooov = blk(Utv, {0, 0, 0, o}, {o, o, o, v}), uovvv = blk(Utv, {0, o, o, o}, {o, v, v, v}),
                     uovov = blk(Utv, {0, o, 0, o}, {o, v, o, v}), uvvvv = blk(Utv, {o, o, o, o}, {v, v, v, v}),
                     uoooo = blk(Utv, {0, 0, 0, 0}, {o, o, o, o}), uovoo = blk(Utv, {0, o, 0, 0}, {o, v, o, o}),
                     uvvov = blk(Utv, {o, o, 0, o}, {v, v, o, v});
            const TV C0v = scal(C0), E0v = scal(E0), C1v = tens(C1, {v, o}), C2v = tens(C2, {v, v, o, o});
            // C0 = 1 + E0 + E0^2/2 + sum fov fvo^T / 2 + sum oovv vvoo / 8  (PCCCI.f90:144-162)
            PHF_TRY(ew(x, "->", ONE, E0v, nullptr, ZERO, C0v));
            PHF_TRY(ew(x, ",->", mkz(0.5), E0v, &E0v, ONE, C0v));
            PHF_TRY(ew(x, "->", ONE, ones1, nullptr, ONE, C0v));
            PHF_TRY(ein(x, "ia,ai->", mkz(0.5), fov, fvo, ONE, C0v));
            PHF_TRY(ein(x, "ijab,abij->", mkz(0.125), uoovv, uvvoo, ONE, C0v));
            // C1 (PCCCI.f90:149, 163-191); "oovv" there holds vvoo transposed after :167
            PHF_TRY(ew(x, "ai->ai", ONE, fvo, nullptr, ZERO, C1v));
            PHF_TRY(ew(x, "ai,->ai", ONE, fvo, &E0v, ONE, C1v));
            PHF_TRY(ein(x, "ak,ki->ai", mkz(-0.5), fvo, foo, ONE, C1v));
            PHF_TRY(ein(x, "ab,bi->ai", mkz(0.5), fvv, fvo, ONE, C1v));
            PHF_TRY(ein(x, "abij,ijkb->ak", mkz(-0.25), uvvoo, uooov, ONE, C1v));
            PHF_TRY(ein(x, "jabc,bckj->ak", mkz(-0.25), uovvv, uvvoo, ONE, C1v));
            PHF_TRY(ein(x, "abij,jb->ai", mkz(0.5), uvvoo, fov, ONE, C1v));
            PHF_TRY(ein(x, "jaib,bj->ai", mkz(-0.5), uovov, fvo, ONE, C1v));
            // C2 (PCCCI.f90:150, 196-275): the C2tmp terms go straight into C2(a,b,i,j)
            PHF_TRY(ew(x, "abij->abij", mkz(0.25), uvvoo, nullptr, ZERO, C2v));
            PHF_TRY(ew(x, "abij,->abij", mkz(0.25), uvvoo, &E0v, ONE, C2v));
            PHF_TRY(ew(x, "aj,bi->abij", mkz(-0.5), fvo, &fvo, ONE, C2v));
            PHF_TRY(ein(x, "acjk,kbic->abij", mkz(0.5), uvvoo, uovov, ONE, C2v));
            PHF_TRY(ein(x, "cdij,abcd->abij", mkz(1.0 / 16), uvvoo, uvvvv, ONE, C2v));
            PHF_TRY(ein(x, "klij,abkl->abij", mkz(1.0 / 16), uoooo, uvvoo, ONE, C2v));
            PHF_TRY(ein(x, "abik,kj->abij", mkz(-0.25), uvvoo, foo, ONE, C2v));
            PHF_TRY(ein(x, "cbij,ac->abij", mkz(0.25), uvvoo, fvv, ONE, C2v));
            PHF_TRY(ein(x, "kbij,ak->abij", mkz(-0.25), uovoo, fvo, ONE, C2v));
            PHF_TRY(ein(x, "abic,cj->abij", mkz(0.25), uvvov, fvo, ONE, C2v));
            // CI2CC (PCCCI.f90:72-98): W0 = C0, W1 = C1/C0, W2 = ASymm2(C2/C0 - W1 W1 / 2)
            recip_kernel<<<(bc + NT - 1) / NT, NT, 0, st>>>(bc, C0, rC0);
            ++g_launches;
            PHF_CHECK_LAUNCH();
            const TV rC0v = scal(rC0), W0v = scal(W0), W1v = tens(W1, {v, o}), W2v = tens(W2, {v, v, o, o}),
                     tmpv = tens(tmp, {v, v, o, o});
            PHF_TRY(ew(x, "ai,->ai", ONE, C1v, &rC0v, ZERO, W1v));
            PHF_TRY(ew(x, "abij,->abij", ONE, C2v, &rC0v, ZERO, tmpv));
            PHF_TRY(ew(x, "ai,bj->abij", mkz(-0.5), W1v, &W1v, ONE, tmpv));
            PHF_TRY(ew(x, "abij->abij", ONE, tmpv, nullptr, ZERO, C2v));  // X2 = T - T(ij swapped)
            PHF_TRY(ew(x, "abji->abij", mkz(-1), tmpv, nullptr, ONE, C2v));
            PHF_TRY(ew(x, "abij->abij", ONE, C2v, nullptr, ZERO, W2v));   // W2 = X2 - X2(ab swapped)
            PHF_TRY(ew(x, "baij->abij", mkz(-1), C2v, nullptr, ONE, W2v));
            // DSTT2 (FPUCC_Tools.f90:714-715): W0 = C0 U0, W1 += U1
            const TV U0v = scal(U0);
            PHF_TRY(ew(x, ",->", ONE, C0v, &U0v, ZERO, W0v));
            PHF_TRY(ew(x, "ai->ai", ONE, U1v, nullptr, ONE, W1v));

            // ---- BuildKernSD (FPUCC_Tools.f90:291-436) with U1t = W1, U2t = W2
            const TV Ovl2v = tens(Ovl2, {v, v, o, o}), EO0v = scal(EO0), EO1v = tens(EO1, {v, o}),
                     EO2v = tens(EO2, {v, v, o, o});
            // Ovl2 = W2 + W1(a,i) W1(b,j) - W1(b,i) W1(a,j)   (:348-350)
            PHF_TRY(ew(x, "abij->abij", ONE, W2v, nullptr, ZERO, Ovl2v));
            PHF_TRY(ew(x, "ai,bj->abij", ONE, W1v, &W1v, ONE, Ovl2v));
            PHF_TRY(ew(x, "bi,aj->abij", mkz(-1), W1v, &W1v, ONE, Ovl2v));
            // CCEnergy (CCRes.f90:9-29) + E_SCF: sum F_ia W1_ai + sum <ij||ab> Ovl2(a,b,i,j) / 4
            PHF_TRY(ein(x, "ia,ai->", ONE, sh(Fov_s), W1v, ZERO, EO0v));
            PHF_TRY(ein(x, "ijab,abij->", mkz(0.25), Hoovv, Ovl2v, ONE, EO0v));
            PHF_TRY(ew(x, "->", ONE, scal(escf, false), nullptr, ONE, EO0v));
            if (sz) PHF_TRY(mask_sz(x, Ovl2v, o, v, nao));  // :356-358

            // CCItms (CCRes.f90:355-537)
            const TV itm1v = tens(itm1, {v, v, o, o}), tauv = tens(tau, {v, v, o, o}), tbv = tens(tb, {v, v, o, o}),
                     itm4v = tens(itm4, {v, v, o, o}), Fvvv = tens(Fvv, {v, v}), Foov = tens(Foo, {o, o}),
                     Fovv = tens(Fov, {o, v}), Wov = tens(Wo, {o, o, o, o}), Wvv = tens(Wv, {v, v, v, v}),
                     Wovvov = tens(Wovvo, {o, v, v, o});
            PHF_TRY(ew(x, "ai,bj->abij", ONE, W1v, &W1v, ZERO, itm1v));           // :397-405
            PHF_TRY(ew(x, "abij->abij", mkz(0.5), W2v, nullptr, ZERO, itm4v));    // :407
            PHF_TRY(ew(x, "abij->abij", ONE, itm1v, nullptr, ONE, itm4v));
            // APerm(itm1, 1) then APerm(itm1, 2) (:408-409) into tmp
            PHF_TRY(ew(x, "abij->abij", ONE, itm1v, nullptr, ZERO, C2v));
            PHF_TRY(ew(x, "baij->abij", mkz(-1), itm1v, nullptr, ONE, C2v));
            PHF_TRY(ew(x, "abij->abij", ONE, C2v, nullptr, ZERO, tmpv));
            PHF_TRY(ew(x, "abji->abij", mkz(-1), C2v, nullptr, ONE, tmpv));
            PHF_TRY(ew(x, "abij->abij", ONE, W2v, nullptr, ZERO, tauv));          // tau = T2 + itm1/2 (:410)
            PHF_TRY(ew(x, "abij->abij", mkz(0.5), tmpv, nullptr, ONE, tauv));
            PHF_TRY(ew(x, "abij->abij", ONE, W2v, nullptr, ZERO, tbv));           // tb = T2 + itm1/4 (:411)
            PHF_TRY(ew(x, "abij->abij", mkz(0.25), tmpv, nullptr, ONE, tbv));
            // Fvv (:418-433)
            PHF_TRY(ew(x, "ab->ab", ONE, sh(Fvv_s), nullptr, ZERO, Fvvv));
            PHF_TRY(ein(x, "ai,ib->ab", mkz(-0.5), W1v, sh(Fov_s), ONE, Fvvv));
            PHF_TRY(ein(x, "ci,aibc->ab", ONE, W1v, Hvovv, ONE, Fvvv));
            PHF_TRY(ein(x, "abij,ijcb->ac", mkz(-0.5), tbv, Hoovv, ONE, Fvvv));
            // Foo (:436-449)
            PHF_TRY(ew(x, "ij->ij", ONE, sh(Foo_s), nullptr, ZERO, Foov));
            PHF_TRY(ein(x, "ia,aj->ij", mkz(0.5), sh(Fov_s), W1v, ONE, Foov));
            PHF_TRY(ein(x, "ak,ikja->ij", ONE, W1v, Hooov, ONE, Foov));
            PHF_TRY(ein(x, "ikcb,cbjk->ij", mkz(0.5), Hoovv, tbv, ONE, Foov));
            // Fov (:453-461)
            PHF_TRY(ew(x, "ia->ia", ONE, sh(Fov_s), nullptr, ZERO, Fovv));
            PHF_TRY(ein(x, "bj,ijab->ia", ONE, W1v, Hoovv, ONE, Fovv));
            // Woooo (:465-471)
            PHF_TRY(ew(x, "ijkl->ijkl", ONE, Hoooo, nullptr, ZERO, Wov));
            PHF_TRY(ein(x, "ijab,abkl->ijkl", mkz(0.25), Hoovv, tauv, ONE, Wov));
            PHF_TRY(ein(x, "ijka,al->ijkl", ONE, Hooov, W1v, ONE, Wov));
            PHF_TRY(ein(x, "ijla,ak->ijkl", mkz(-1), Hooov, W1v, ONE, Wov));
            // Wvvvv (:474-496)
            PHF_TRY(ew(x, "abcd->abcd", ONE, Hvvvv, nullptr, ZERO, Wvv));
            PHF_TRY(ein(x, "cdij,ijab->cdab", mkz(0.25), tauv, Hoovv, ONE, Wvv));
            PHF_TRY(ein(x, "aicd,bi->abcd", mkz(-1), Hvovv, W1v, ONE, Wvv));
            PHF_TRY(ein(x, "bicd,ai->abcd", ONE, Hvovv, W1v, ONE, Wvv));
            // Wovvo (:502-530)
            PHF_TRY(ew(x, "iabj->iabj", ONE, Hovvo, nullptr, ZERO, Wovvov));
            PHF_TRY(ein(x, "iabc,cj->iabj", ONE, Hovvv, W1v, ONE, Wovvov));
            PHF_TRY(ein(x, "ikcj,bk->ibcj", mkz(-1), Hoovo, W1v, ONE, Wovvov));
            PHF_TRY(ein(x, "dbjk,ikcd->ibcj", mkz(-1), itm4v, Hoovv, ONE, Wovvov));

            // CCRes12 (CCRes.f90:164-353): r1 and res2 (res2 collects r2tmp transposed, then + H2 vvoo)
            const TV r1v = tens(r1, {v, o}), res2v = tens(res2, {v, v, o, o}), itm2v = tens(itm2, {o, o, v, v}),
                     itm4bv = tens(itm4b, {o, o, o, v}), itm1pv = tens(itm1p, {v, v}), itm3pv = tens(itm3p, {o, o});
            PHF_TRY(ew(x, "ai->ai", ONE, sh(Fvo_s), nullptr, ZERO, r1v));                 // :213
            PHF_TRY(ein(x, "ab,bi->ai", ONE, Fvvv, W1v, ONE, r1v));
            PHF_TRY(ein(x, "ak,ki->ai", mkz(-1), W1v, Foov, ONE, r1v));
            PHF_TRY(ein(x, "jb,abij->ai", ONE, Fovv, W2v, ONE, r1v));                     // :217
            PHF_TRY(ein(x, "bj,ajib->ai", ONE, W1v, Hvoov, ONE, r1v));                    // :218
            PHF_TRY(ein(x, "abjk,jkib->ai", mkz(-0.5), W2v, Hooov, ONE, r1v));            // :220-226
            PHF_TRY(ein(x, "ajcb,cbij->ai", mkz(0.5), Hvovv, W2v, ONE, r1v));             // :227-233
            PHF_TRY(ew(x, "abij->abij", ONE, Hvvoo, nullptr, ZERO, res2v));               // r2 (:237)
            // itm1 = Fvv - W1 Fov / 2; r2tmp += APerm2(sum_c t2(a,c,i,j) itm1(b,c))   (:239-251)
            PHF_TRY(ew(x, "ab->ab", ONE, Fvvv, nullptr, ZERO, itm1pv));
            PHF_TRY(ein(x, "ai,ib->ab", mkz(-0.5), W1v, Fovv, ONE, itm1pv));
            PHF_TRY(ein(x, "acij,bc->abij", ONE, W2v, itm1pv, ONE, res2v));
            PHF_TRY(ein(x, "bcij,ac->abij", mkz(-1), W2v, itm1pv, ONE, res2v));
            // itm3 = Foo + Fov W1 / 2; r2tmp -= APerm1(sum_k t2(a,b,i,k) itm3(k,j))   (:254-267)
            PHF_TRY(ew(x, "ij->ij", ONE, Foov, nullptr, ZERO, itm3pv));
            PHF_TRY(ein(x, "ia,aj->ij", mkz(0.5), Fovv, W1v, ONE, itm3pv));
            PHF_TRY(ein(x, "abik,kj->abij", mkz(-1), W2v, itm3pv, ONE, res2v));
            PHF_TRY(ein(x, "abjk,ki->abij", ONE, W2v, itm3pv, ONE, res2v));
            // itm4(k,j,i,b) = sum_c W1(c,k) H2(i,b,c,j); itm2(k,j,a,b) = -sum_i itm4(k,j,i,b) W1(a,i)
            // + sum_kc t2(a,c,i,k) Wovvo(k,b,c,j); r2tmp += APerm1 APerm2 itm2   (:270-306)
            PHF_TRY(ein(x, "ck,ibcj->kjib", ONE, W1v, Hovvo, ZERO, itm4bv));
            PHF_TRY(ein(x, "kjib,ai->kjab", mkz(-1), itm4bv, W1v, ZERO, itm2v));
            PHF_TRY(ein(x, "acik,kbcj->ijab", ONE, W2v, Wovvov, ONE, itm2v));
            PHF_TRY(ew(x, "ijab->abij", ONE, itm2v, nullptr, ONE, res2v));
            PHF_TRY(ew(x, "jiab->abij", mkz(-1), itm2v, nullptr, ONE, res2v));
            PHF_TRY(ew(x, "ijba->abij", mkz(-1), itm2v, nullptr, ONE, res2v));
            PHF_TRY(ew(x, "jiba->abij", ONE, itm2v, nullptr, ONE, res2v));
            // + tau Wvvvv / 2 + Woooo tau / 2   (:308-322)
            PHF_TRY(ein(x, "cdij,abcd->abij", mkz(0.5), tauv, Wvv, ONE, res2v));
            PHF_TRY(ein(x, "klij,abkl->abij", mkz(0.5), Wov, tauv, ONE, res2v));
            // + APerm1(sum_c W1(c,i) H2(a,b,c,j)) - APerm2(sum_k H2(k,b,i,j) W1(a,k))   (:327-348)
            PHF_TRY(ein(x, "ci,abcj->abij", ONE, W1v, Hvvvo, ONE, res2v));
            PHF_TRY(ein(x, "cj,abci->abij", mkz(-1), W1v, Hvvvo, ONE, res2v));
            PHF_TRY(ein(x, "kbij,ak->abij", mkz(-1), Hovoo, W1v, ONE, res2v));
            PHF_TRY(ein(x, "kaij,bk->abij", ONE, Hovoo, W1v, ONE, res2v));

            // EOvl1 = r1 + W1 EOvl0 (:392), EOvl2 (:416-421)
            PHF_TRY(ew(x, "ai->ai", ONE, r1v, nullptr, ZERO, EO1v));
            PHF_TRY(ew(x, "ai,->ai", ONE, W1v, &EO0v, ONE, EO1v));
            PHF_TRY(ew(x, "abij->abij", ONE, res2v, nullptr, ZERO, EO2v));
            PHF_TRY(ew(x, "abij,->abij", ONE, Ovl2v, &EO0v, ONE, EO2v));
            PHF_TRY(ew(x, "ai,bj->abij", ONE, W1v, &r1v, ONE, EO2v));
            PHF_TRY(ew(x, "bi,aj->abij", mkz(-1), W1v, &r1v, ONE, EO2v));
            PHF_TRY(ew(x, "bj,ai->abij", ONE, W1v, &r1v, ONE, EO2v));
            PHF_TRY(ew(x, "aj,bi->abij", mkz(-1), W1v, &r1v, ONE, EO2v));
            if (g.trunode == 3) {  // EvalKernel :577-581: eps0 += the (T) energy of (W1, W2) after BuildKernSD
                const TV Hvvvo_ = blk(H2v, {o, o, o, 0}, {v, v, v, o});
                for (int s0 = 0; s0 < bc; s0 += nsubT) {
                    const int ns = std::min(nsubT, bc - s0);
                    x.npts = ns;
                    const size_t mark = x.used;
                    TV W2s = W2v, W1s = W1v;
                    W2s.p += s0 * W2v.ps;
                    W1s.p += s0 * W1v.ps;
                    PHF_TRY(check_view(x, tpart, ntri, 1, 1, 0, ns, ntri, 1, 0, "(T) parts"));
                    PHF_TRY(check_view(x, W2s.p, vvoo, 1, 1, 0, ns, W2v.ps, 1, 0, "(T) T2"));
                    PHF_TRY(check_view(x, W1s.p, vo, 1, 1, 0, ns, W1v.ps, 1, 0, "(T) T1"));
                    PHF_TRY(check_tv(x, Hvvvo_, 1, "(T) <vv||vo>"));
                    PHF_TRY(check_tv(x, Hovoo, 1, "(T) <ov||oo>"));
                    PHF_TRY(check_tv(x, Hvvoo, 1, "(T) <vv||oo>"));
                    PHF_TRY(check_tv(x, Fvo_s, 1, "(T) F_vo"));
                    TriplesArgs ta{o, v, trid, Wtrip, o3v3, W1s.p, W1v.ps, W2s.p, W2v.ps, Hvvoo.p, Fvo_s.p, F, M, tpart,
                                   ntri};
                    if (fusedT) {
                        const size_t sm = (size_t)o * o * o * sizeof(zc);
                        PHF_CUDA(cudaFuncSetAttribute(triples_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)sm));
                        triples_fused_kernel<<<dim3((unsigned)ntri, (unsigned)ns), NT, sm, st>>>(ta, Hvvvo_.p, Hovoo.p);
                    } else {
                        // W(x,b,c,a,y,z) = sum_d <bc||dx> T2(a,d,y,z) - sum_l T2(b,c,x,l) <la||yz>  (get_wv :62-63) as
                        // one GEMM with k = v + o: rows (x,b,c) of A = [<bc||dx> | -T2(b,c,x,l)], columns (a,y,z) of
                        // B = [T2(a,d,y,z); <la||yz>]
                        const long long mT = (long long)o * v * v, nT = (long long)v * o * o, kT = (long long)v + o;
                        TV Ad = tens(Aop, {o, v, v, v}), Al = tens(Aop, {o, v, v, o}), Bd = tens(Bop, {v, v, o, o}),
                           Bl = tens(Bop, {o, v, o, o});
                        Ad.ps = Al.ps = mT * kT;
                        Bd.ps = Bl.ps = kT * nT;
                        Al.p += mT * v;  // A: column-major m x k, d columns then l columns
                        Ad.st[3] = Al.st[3] = mT;
                        Bl.p += v;       // B: column-major k x n, d rows then l rows
                        Bd.st[0] = Bl.st[0] = 1;
                        Bd.st[1] = Bl.st[1] = kT;
                        Bd.st[2] = Bl.st[2] = kT * v;
                        Bd.st[3] = Bl.st[3] = kT * v * o;
                        PHF_TRY(ew(x, "bcdx->xbcd", ONE, Hvvvo_, nullptr, ZERO, Ad));
                        PHF_TRY(ew(x, "bcxl->xbcl", mkz(-1), W2s, nullptr, ZERO, Al));
                        PHF_TRY(ew(x, "adyz->dayz", ONE, W2s, nullptr, ZERO, Bd));
                        PHF_TRY(ew(x, "layz->layz", ONE, Hovoo, nullptr, ZERO, Bl));
                        PHF_TRY(check_view(x, Aop, mT, kT, 1, mT, ns, mT * kT, 1, 0, "(T) A"));
                        PHF_TRY(check_view(x, Bop, kT, nT, 1, kT, ns, kT * nT, 1, 0, "(T) B"));
                        PHF_TRY(check_view(x, Wtrip, mT, nT, 1, mT, ns, o3v3, 1, 0, "(T) W"));
                        PHF_TRY(zgemm_strided((int)mT, (int)nT, (int)kT, ns, 1, ONE, View{Aop, 1, mT, mT * kT},
                                              View{Bop, 1, kT, kT * nT}, ZERO, OutView{Wtrip, 1, mT, o3v3}, nullptr, st));
                        g_pcc_flops += 8.0 * (double)mT * (double)nT * (double)kT * ns;
                        triples_kernel<<<dim3((unsigned)ntri, (unsigned)ns), NT, 0, st>>>(ta);
                    }
                    ++g_launches;
                    PHF_CHECK_LAUNCH();
                    TV pv;
                    pv.p = tpart;
                    pv.nd = 1;
                    pv.dim[0] = (int)ntri;
                    pv.st[0] = 1;
                    pv.ps = ntri;
                    PHF_TRY(ein(x, "t,t->", mkz(0.5), pv, ones_v((int)ntri), ONE, scal(EO0 + s0)));
                    x.used = mark;
                }
                x.npts = bc;
            }
            if (sz) {  // BuildKernSD :329-332, :398-400, :426-428 and EvalKernel :584-589
                PHF_TRY(mask_sz(x, W1v, o, v, nao));
                PHF_TRY(mask_sz(x, EO1v, o, v, nao));
                PHF_TRY(mask_sz(x, EO2v, o, v, nao));
            }
            // sums over the chunk's points in point order, lambda0 = W0 folded into the weight
            // (eps0, eps1, eps2, lambda1, lambda2 are lambda0 times EOvl0, EOvl1, EOvl2, Ovl1, Ovl2, :590-596)
            const TV swv = scal(sw), wtv = [&] {
                TV t;
                t.p = wtd + w0;
                t.ps = 1;
                return t;
            }();
            PHF_TRY(ew(x, ",->", ONE, wtv, &W0v, ZERO, swv));
            if (pass) PHF_TRY(ew(x, "->", mkz(g.fk[1].re, g.fk[1].im), swv, nullptr, ZERO, swv));
            auto pt = [&](TV t) {  // the point as the last index of a per-point tensor
                t.dim[t.nd] = bc;
                t.st[t.nd] = t.ps;
                ++t.nd;
                t.ps = 0;
                return t;
            };
            auto sum_pts = [&](const char *spec, const TV &wv, const TV &val, zc *dst, std::initializer_list<int> dims) {
                TV d = tens(dst, dims, false);
                return ein(x, spec, ONE, pt(wv), pt(val), ONE, d, 1);
            };
            PHF_TRY(sum_pts("w,w->", swv, EO0v, aE0, {}));
            PHF_TRY(ew(x, ",->", pass ? mkz(g.fk[1].re, g.fk[1].im) : ONE, wtv, &W0v, ZERO, tens(det2, {}), bc));
            PHF_TRY(sum_pts("w,w->", tens(det2, {}), ones1, aL0, {}));
            PHF_TRY(sum_pts("w,aiw->ai", swv, EO1v, aE1, {v, o}));
            PHF_TRY(sum_pts("w,aiw->ai", swv, W1v, aL1, {v, o}));
            PHF_TRY(sum_pts("w,abijw->abij", swv, EO2v, aE2, {v, v, o, o}));
            PHF_TRY(sum_pts("w,abijw->abij", swv, Ovl2v, aL2, {v, v, o, o}));
        }
    }
    x.npts = 1;
    if (sz) {  // ProjSz of the sums (:231-234)
        PHF_TRY(mask_sz(x, tens(aE1, {v, o}, false), o, v, nao));
        PHF_TRY(mask_sz(x, tens(aL1, {v, o}, false), o, v, nao));
        PHF_TRY(mask_sz(x, tens(aE2, {v, v, o, o}, false), o, v, nao));
        PHF_TRY(mask_sz(x, tens(aL2, {v, v, o, o}, false), o, v, nao));
    }
    PHF_CUDA(cudaEventRecord(ev1, st));
    std::vector<cd> h((size_t)nacc);
    int hflag = 0;
    PHF_CUDA(cudaMemcpyAsync(h.data(), acc, nacc * sizeof(zc), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    PHF_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    PHF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    g_pcc_ms = ms;
    if (hflag & 1) {
        set_error(PHF_ERR_SINGULAR, "pbarhbarolap: a rotated occupied block or the transform V is exactly singular");
        return PHF_ERR_SINGULAR;
    }
    for (const cd &z : h)
        if (!std::isfinite(z.real()) || !std::isfinite(z.imag()) || (hflag & 2)) {
            set_error(PHF_ERR_NONFINITE, "pbarhbarolap: non-finite result");
            return PHF_ERR_NONFINITE;
        }
    auto put = [&](phf_complex *dst, const cd *src, long long n) {
        for (long long i = 0; i < n; ++i) dst[i] = phf_complex{src[i].real(), src[i].imag()};
    };
    put(eolap0, &h[0], 1);
    put(olap0, &h[1], 1);
    put(eolapex1, &h[2], vo);
    put(olapex1, &h[2 + vo], vo);
    put(eolapex2, &h[2 + 2 * vo], vvoo);
    put(olapex2, &h[2 + 2 * vo + vvoo], vvoo);
    return PHF_OK;
}

}  // namespace phf

extern "C" int phf_pbarhbarolap(phf_complex *olap0, phf_complex *olapex1, phf_complex *olapex2, phf_complex *eolap0,
                                phf_complex *eolapex1, phf_complex *eolapex2, const phf_complex *hone,
                                const phf_complex *htwo, const phf_complex *ref, const phf_complex *t1,
                                const phf_complex *t2, int nocc, int nao, int nso, double enuc, int qj, int sp,
                                const int *npoints, int npg, int ncisp, int ncipg, int ncik, const phf_complex *r1,
                                const phf_complex *r2, const phf_complex *rpg, const phf_complex *rk,
                                const double *roota, const double *rootb, const double *rooty, const double *weightsp,
                                const double *weightpg, const phf_complex *fsp, const phf_complex *fpg,
                                const phf_complex *fk, int trunode, size_t workspace) {
    (void)ref;
    phf::set_error(PHF_OK, "");
    if (!olap0 || !olapex1 || !olapex2 || !eolap0 || !eolapex1 || !eolapex2 || !hone || !htwo || !t1 || !t2 ||
        !npoints || !r1 || !r2 || !rpg || !roota || !rootb || !rooty || !weightsp || !weightpg || !fsp || !fpg || !fk ||
        nso <= 0 || nocc <= 0 || nocc >= nso || npoints[0] <= 0 || npoints[1] <= 0 || npg <= 0 || ncipg <= 0 ||
        qj < 0 || ncisp != 2 * qj + 1 || (ncik != 1 && ncik != 2) || (ncik == 2 && !rk) || (nao != 0 && 2 * nao != nso)) {
        phf::set_error(PHF_ERR_ARG, "phf_pbarhbarolap: missing or inconsistent argument");
        return PHF_ERR_ARG;
    }
    const int t = trunode < 0 ? -trunode : trunode;
    if (t < 1 || t > 3) {  // BuildKernSD STOPs 'ODE truncation type not recognized' (FPUCC_Tools.f90:314)
        phf::set_error(PHF_ERR_ARG, "phf_pbarhbarolap: ODE truncation type not recognized");
        return PHF_ERR_ARG;
    }
    if (nso > phf::kMaxOverlapN) {
        phf::set_error(PHF_ERR_UNSUPPORTED, "phf_pbarhbarolap: nso above the inverse's limit of 112");
        return PHF_ERR_UNSUPPORTED;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        phf::set_error(PHF_ERR_NO_DEVICE, "no CUDA device available");
        return PHF_ERR_NO_DEVICE;
    }
    phf::PccArgs g{hone, htwo, t1, t2, nocc, nso, enuc, qj, sp, npoints, npg, ncisp, ncipg, ncik, r1, r2, rpg, rk,
                   roota, rootb, rooty, weightsp, weightpg, fsp, fpg, fk, trunode, workspace};
    return phf::pbarhbarolap_run(g, olap0, olapex1, olapex2, eolap0, eolapex1, eolapex2);
}

extern "C" int phf_pbarhbarolap_stats(double *device_ms, double *gemm_flops) {
    if (device_ms) *device_ms = phf::g_pcc_ms;
    if (gemm_flops) *gemm_flops = phf::g_pcc_flops;
    return PHF_OK;
}
