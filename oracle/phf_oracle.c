/*
 * CPU oracle for the projected-HF grid kernel -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker and the timed CPU baseline ("port" of the reference's
 * Fortran, which cannot be compiled here: no Fortran compiler, no MPI).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the product library
 * never links it.
 *
 * It restates PHF_fort/PHFTools.f90 in C99 + OpenMP, FP64 complex throughout:
 *   oracle_buildhsg  -- BuildHSG (PHFTools.f90:10-201): loop il, iy, ipg; R = Ref^H (R1 R2 Rpg) Ref
 *                       (ao2mo2 :390-398); RDM (:249-263) with an LU inverse and determinant
 *                       (stand-ins for InvertC/determinantC, Wrappers.f90:195-336: partial pivoting
 *                       on |re|+|im| as LAPACK's izamax); MakeGamma (:310-337); Kernels/Makeh
 *                       (:281-289, :339-348); Gradient (:291-308); weighting and Wigner x point-group
 *                       accumulation (:120-166).  OpenMP over grid points (the reference splits the
 *                       Lebedev index, :79-84), each thread with private accumulators, reduced in
 *                       thread order.
 *   oracle_localg    -- LocalG (PHFTools.f90:203-247).
 * Gamma comes either from the dense HTwo(M,M,M,M) (the reference form), from MO-basis
 * Cholesky vectors Bt(M,M,L) with (ik|jl) = sum_L Bt[ik] Bt[jl] (identical J - K), or
 * (oracle_buildhsg_ex) from the spatial AO-basis vectors B(n,n,L) with the spin blocks of
 * Main_PHF.py:22-29 written out (the same J - K at a quarter of the work; used where the dense
 * HTwo would not fit in host memory).  With fewer grid points than threads the points run one
 * after another and the work inside each point is split over the threads.
 * CmplxConj == 2 is supported.
 *
 * All arrays use the reference's Fortran (column-major) layouts:
 *   HOne(i,j) = hone[i + M*j];  HTwo(i,j,k,l) = htwo[i + M*(j + M*(k + M*l))]
 *   R1(il,i,j) = r1[il + nl*(i + M*j)];  weightsp(il,iy) = w[il + nl*iy]
 *   weightpg(ipg,p,q) = wpg[ipg + npg*(p + ncipg*q)];  Gradmat(m,n,i,j) = g[m + nci*(n + nci*(i + M*j))]
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex zc;

#define IDX2(i, j, ld) ((size_t)(i) + (size_t)(ld) * (size_t)(j))

/* Threads that share the work of ONE grid point: > 1 only when fewer grid points than threads are
 * evaluated (then the points run one after another and the products and the Cholesky sum inside a
 * point are split over the threads); 1 while the points themselves run in parallel. */
static int g_inner = 1;

/* C = op(A) * B, column-major; A is m x k (opA: 0 none, 2 conj-transpose of a k x m array) */
static void zgemm_cm(int m, int n, int k, const zc *A, int lda, int opA, const zc *B, int ldb, zc *C, int ldc)
{
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int j = 0; j < n; ++j) {
        zc *cj = C + (size_t)ldc * j;
        for (int i = 0; i < m; ++i) cj[i] = 0;
        if (opA == 0) {
            for (int p = 0; p < k; ++p) {
                zc b = B[IDX2(p, j, ldb)];
                const zc *ap = A + (size_t)lda * p;
                for (int i = 0; i < m; ++i) cj[i] += ap[i] * b;
            }
        } else {
            for (int i = 0; i < m; ++i) {
                const zc *ai = A + (size_t)lda * i; /* column i of the k x m array */
                zc s = 0;
                for (int p = 0; p < k; ++p) s += conj(ai[p]) * B[IDX2(p, j, ldb)];
                cj[i] = s;
            }
        }
    }
}

/* LU with partial pivoting (pivot = max |re|+|im|), then inverse and determinant.
 * Returns 0, or 1 when a pivot is exactly zero (the reference STOPs there). */
static int zinv_det(int n, const zc *A, zc *Ainv, zc *det, zc *work, int *piv)
{
    memcpy(work, A, sizeof(zc) * (size_t)n * n);
    zc d = 1.0;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = -1.0;
        for (int i = k; i < n; ++i) {
            zc v = work[IDX2(i, k, n)];
            double a = fabs(creal(v)) + fabs(cimag(v));
            if (a > best) { best = a; p = i; }
        }
        piv[k] = p;
        if (p != k) {
            for (int j = 0; j < n; ++j) {
                zc t = work[IDX2(k, j, n)];
                work[IDX2(k, j, n)] = work[IDX2(p, j, n)];
                work[IDX2(p, j, n)] = t;
            }
            d = -d;
        }
        zc akk = work[IDX2(k, k, n)];
        if (akk == 0) { *det = 0; return 1; }
        d *= akk;
        for (int i = k + 1; i < n; ++i) work[IDX2(i, k, n)] /= akk;
        for (int j = k + 1; j < n; ++j) {
            zc akj = work[IDX2(k, j, n)];
            if (akj == 0) continue;
            for (int i = k + 1; i < n; ++i) work[IDX2(i, j, n)] -= work[IDX2(i, k, n)] * akj;
        }
    }
    *det = d;
    /* inverse: solve A X = I column by column with the LU factors */
    for (int c = 0; c < n; ++c) {
        zc *x = Ainv + (size_t)n * c;
        for (int i = 0; i < n; ++i) x[i] = (i == c) ? 1.0 : 0.0;
        for (int k = 0; k < n; ++k) { /* apply the row interchanges */
            int p = piv[k];
            if (p != k) { zc t = x[k]; x[k] = x[p]; x[p] = t; }
        }
        for (int i = 0; i < n; ++i) { /* L y = x (unit lower) */
            zc s = x[i];
            for (int k = 0; k < i; ++k) s -= work[IDX2(i, k, n)] * x[k];
            x[i] = s;
        }
        for (int i = n - 1; i >= 0; --i) { /* U z = y */
            zc s = x[i];
            for (int k = i + 1; k < n; ++k) s -= work[IDX2(i, k, n)] * x[k];
            x[i] = s / work[IDX2(i, i, n)];
        }
    }
    return 0;
}

static double wigner_small_d(int j, int n, int m, double beta)
{
    double fj[64];
    fj[0] = 1.0;
    for (int i = 1; i < 64; ++i) fj[i] = fj[i - 1] * i;
    double pre = sqrt(fj[j + n] * fj[j - n] * fj[j + m] * fj[j - m]);
    int smax = (j + m < j - n) ? j + m : j - n;
    int smin = (m - n > 0) ? m - n : 0;
    double acc = 0.0;
    for (int s = smin; s <= smax; ++s) {
        int p1 = n - m + s, p2 = 2 * j + m - n - 2 * s, p3 = n - m + 2 * s;
        double num = ((p1 & 1) ? -1.0 : 1.0) * pow(cos(beta / 2), p2) * pow(sin(beta / 2), p3);
        double den = fj[j + m - s] * fj[s] * fj[n - m + s] * fj[j - n - s];
        acc += num / den;
    }
    return pre * acc;
}

/* Wignerfac (PHFTools.f90:350-376) */
static zc wignerfac(int j, int n, int m, double alpha, double beta, double gamma)
{
    return cexp(-I * n * alpha) * wigner_small_d(j, n, m, beta) * cexp(-I * m * gamma);
}

typedef struct {
    int M, N, L;
    const zc *hone, *htwo, *bt;
    const double *bs; /* spatial Cholesky vectors B(p,q,L) = bs[p + n*(q + n*L)] in the AO basis */
    const zc *ref;    /* Ref (M x M): MO = AO Ref, for the spatial form */
} ham_t;

/* C (n x n complex) = A (n x n real) * B (n x n complex, leading dimension ldb), column-major */
static void dz_gemm(int n, const double *A, const zc *B, int ldb, zc *C)
{
    for (int j = 0; j < n; ++j) {
        zc *cj = C + (size_t)n * j;
        for (int i = 0; i < n; ++i) cj[i] = 0;
        for (int p = 0; p < n; ++p) {
            const zc b = B[(size_t)p + (size_t)ldb * j];
            const double *ap = A + (size_t)n * p;
            for (int i = 0; i < n; ++i) cj[i] += ap[i] * b;
        }
    }
}

/* Gamma from spatial Cholesky vectors (the same J - K as the MO-basis form, with the spin
 * structure B~_L = blockdiag(B_L, B_L) of Main_PHF.py:22-29 used explicitly):
 *   rho_AO = Ref rho Ref^H;  P = rho_aa + rho_bb;  d_L = tr(B_L P)
 *   J = sum_L d_L B_L on both spin diagonal blocks;  K_st = sum_L B_L rho_st B_L (four spin blocks)
 *   gama = Ref^H (J - K) Ref
 * The L sum is split over g_inner threads in contiguous ranges, added in thread order. */
static void make_gamma_spatial(const ham_t *H, const zc *rho, zc *gama, zc *tmp)
{
    const int M = H->M, n = M / 2, L = H->L, nt = g_inner;
    const size_t MM = (size_t)M * M, nn = (size_t)n * n;
    const zc *ref = H->ref;
    zc *rao = malloc(sizeof(zc) * MM), *part = calloc((size_t)nt * 5 * nn, sizeof(zc));
    zgemm_cm(M, M, M, ref, M, 0, rho, M, tmp, M); /* Ref rho */
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
    for (int j = 0; j < M; ++j) /* rao = (Ref rho) Ref^H */
        for (int i = 0; i < M; ++i) {
            zc a = 0;
            for (int p = 0; p < M; ++p) a += tmp[IDX2(i, p, M)] * conj(ref[IDX2(j, p, M)]);
            rao[IDX2(i, j, M)] = a;
        }
#pragma omp parallel num_threads(nt) if (nt > 1)
    {
        int t = 0;
#ifdef _OPENMP
        if (nt > 1) t = omp_get_thread_num();
#endif
        const int l0 = (int)((long long)L * t / nt), l1 = (int)((long long)L * (t + 1) / nt);
        zc *Jp = part + (size_t)t * 5 * nn, *Kp = Jp + nn;
        zc *T = malloc(sizeof(zc) * nn), *U = malloc(sizeof(zc) * nn);
        for (int l = l0; l < l1; ++l) {
            const double *b = H->bs + (size_t)l * nn;
            zc d = 0;
            for (int q = 0; q < n; ++q)
                for (int p = 0; p < n; ++p) d += b[IDX2(p, q, n)] * (rao[IDX2(q, p, M)] + rao[IDX2(n + q, n + p, M)]);
            for (size_t e = 0; e < nn; ++e) Jp[e] += d * b[e];
            for (int st = 0; st < 4; ++st) {
                const int sg = st >> 1, tu = st & 1;
                dz_gemm(n, b, rao + (size_t)sg * n + (size_t)M * tu * n, M, T); /* B rho_st */
                for (int j = 0; j < n; ++j)                                    /* (B rho_st) B */
                    for (int i = 0; i < n; ++i) U[IDX2(i, j, n)] = 0;
                for (int j = 0; j < n; ++j)
                    for (int p = 0; p < n; ++p) {
                        const double bpj = b[IDX2(p, j, n)];
                        const zc *tp = T + (size_t)n * p;
                        zc *uj = U + (size_t)n * j;
                        for (int i = 0; i < n; ++i) uj[i] += tp[i] * bpj;
                    }
                zc *Ks = Kp + (size_t)st * nn;
                for (size_t e = 0; e < nn; ++e) Ks[e] += U[e];
            }
        }
        free(T);
        free(U);
    }
    /* Gamma_AO = blockdiag(J, J) - K, partial sums added in thread order */
    for (size_t e = 0; e < MM; ++e) rao[e] = 0;
    for (int t = 0; t < nt; ++t) {
        const zc *Jp = part + (size_t)t * 5 * nn, *Kp = Jp + nn;
        for (int st = 0; st < 4; ++st) {
            const int sg = st >> 1, tu = st & 1;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    zc v = -Kp[(size_t)st * nn + IDX2(i, j, n)];
                    if (sg == tu) v += Jp[IDX2(i, j, n)];
                    rao[IDX2(sg * n + i, tu * n + j, M)] += v;
                }
        }
    }
    zgemm_cm(M, M, M, rao, M, 0, ref, M, tmp, M); /* Gamma_AO Ref */
    zgemm_cm(M, M, M, ref, M, 2, tmp, M, gama, M); /* Ref^H Gamma_AO Ref */
    free(rao);
    free(part);
}

/* gama_ik = sum_jl H2_ijkl rho_lj (MakeGamma) or the J - K Cholesky form */
static void make_gamma(const ham_t *H, const zc *rho, zc *gama, zc *tmp)
{
    const int M = H->M;
    if (H->htwo) {
        for (int k = 0; k < M; ++k)
            for (int i = 0; i < M; ++i) {
                zc s = 0;
                for (int l = 0; l < M; ++l) {
                    const zc *h = H->htwo + (size_t)i + (size_t)M * ((size_t)M * ((size_t)k + (size_t)M * l));
                    const zc *r = rho + l; /* rho(l, j) = rho[l + M j] */
                    for (int j = 0; j < M; ++j) s += h[(size_t)M * j] * r[(size_t)M * j];
                }
                gama[IDX2(i, k, M)] = s;
            }
        return;
    }
    if (H->bs) {
        make_gamma_spatial(H, rho, gama, tmp);
        return;
    }
    /* Cholesky: J_ik = sum_L Bt_L[ik] tr(Bt_L rho); K = sum_L Bt_L rho Bt_L */
    memset(gama, 0, sizeof(zc) * (size_t)M * M);
    for (int L = 0; L < H->L; ++L) {
        const zc *b = H->bt + (size_t)L * M * M;
        zc d = 0;
        for (int j = 0; j < M; ++j)
            for (int l = 0; l < M; ++l) d += b[IDX2(j, l, M)] * rho[IDX2(l, j, M)];
        zgemm_cm(M, M, M, b, M, 0, rho, M, tmp, M);               /* tmp = B rho */
        for (int k = 0; k < M; ++k)
            for (int i = 0; i < M; ++i) {
                zc s = 0;
                for (int p = 0; p < M; ++p) s += tmp[IDX2(i, p, M)] * b[IDX2(p, k, M)];
                gama[IDX2(i, k, M)] += d * b[IDX2(i, k, M)] - s;
            }
    }
}

/* Makeh: sum(H1^T * rho) + sum(gama * rho^T)/2 */
static zc makeh(int M, const zc *h1, const zc *gama, const zc *rho)
{
    zc h = 0, g = 0;
    for (int j = 0; j < M; ++j)
        for (int i = 0; i < M; ++i) {
            h += h1[IDX2(j, i, M)] * rho[IDX2(i, j, M)];
            g += gama[IDX2(i, j, M)] * rho[IDX2(j, i, M)];
        }
    return h + g / 2.0;
}

typedef struct {
    zc *R, *Rt, *Rt2, *tmp, *Mm, *Minv, *work, *rho, *gama, *g, *t2;
    int *piv;
} scratch_t;

/* RDM (:249-263) / RDMConj (:265-279) with ket = conjugated when conj_ket, bra = conjugated when conj_bra */
static int rdm(int M, int N, const zc *R, const zc *mo, int conj_bra, int conj_ket, scratch_t *s, zc *rho, zc *det)
{
    zc *bra = s->t2, *ket = s->t2 + (size_t)M * N;
    for (size_t i = 0; i < (size_t)M * N; ++i) {
        bra[i] = conj_bra ? conj(mo[i]) : mo[i];
        ket[i] = conj_ket ? conj(mo[i]) : mo[i];
    }
    zgemm_cm(M, N, M, R, M, 0, ket, M, s->tmp, M);           /* tmp = R ket */
    zgemm_cm(N, N, M, bra, M, 2, s->tmp, M, s->Mm, N);       /* Mm = bra^H tmp */
    if (zinv_det(N, s->Mm, s->Minv, det, s->work, s->piv)) return 1;
    zc *t3 = s->Rt2;                                          /* M x N */
    zgemm_cm(M, N, N, s->tmp, M, 0, s->Minv, N, t3, M);      /* tmp Minv */
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int j = 0; j < M; ++j)                               /* rho = t3 bra^H */
        for (int i = 0; i < M; ++i) {
            zc acc = 0;
            for (int p = 0; p < N; ++p) acc += t3[IDX2(i, p, M)] * conj(bra[IDX2(j, p, M)]);
            rho[IDX2(i, j, M)] = acc;
        }
    return 0;
}

/* Gradient (:291-308): det * [(I - rho)(H1 + gama) rho + h rho] */
static void gradient(const ham_t *H, const zc *gama, const zc *rho, zc det, scratch_t *s, zc *g)
{
    const int M = H->M;
    zc h = makeh(M, H->hone, gama, rho);
    zc *F = s->Rt, *FR = s->R;
    for (size_t i = 0; i < (size_t)M * M; ++i) F[i] = H->hone[i] + gama[i];
    zgemm_cm(M, M, M, F, M, 0, rho, M, FR, M);                /* F rho */
#pragma omp parallel for schedule(static) num_threads(g_inner) if (g_inner > 1)
    for (int j = 0; j < M; ++j)
        for (int i = 0; i < M; ++i) {
            zc acc = FR[IDX2(i, j, M)];
            for (int p = 0; p < M; ++p) acc -= rho[IDX2(i, p, M)] * FR[IDX2(p, j, M)];
            g[IDX2(i, j, M)] = (acc + h * rho[IDX2(i, j, M)]) * det;
        }
}

/* bs != NULL: Gamma from the spatial Cholesky vectors bs (AO basis, n = nso/2, nchol of them)
 * through make_gamma_spatial, with the MO basis given by ref; else from htwo or bt. */
int oracle_buildhsg_ex(const zc *hone, const zc *htwo, const zc *bt, const double *bs, int nchol, const zc *ref,
                       const zc *z, const int *ngrid, int nci, int cmplxconj, int ncisp, int nocc, const zc *r1,
                       const zc *r2, const zc *rpg, const double *weightsp, const double *weightpg,
                       const double *roota, const double *rootb, const double *rooty, int qj, int sp, int npg,
                       int ncipg, int nso, const int *omega_list, int n_omega, int nthreads, zc *hmat, zc *smat,
                       zc *gradmat, zc *rdmmat)
{
    const int M = nso, N = nocc, nl = ngrid[0], ny = ngrid[1];
    const size_t MM = (size_t)M * M;
    const int nw = 2 * qj + 1;
    if (nw != ncisp && sp == 1) return -1;
    ham_t H = {M, N, nchol, hone, htwo, bt, bs, ref};
    zc *newmo = calloc((size_t)M * N, sizeof(zc));
    for (int i = 0; i < N; ++i) newmo[IDX2(i, i, M)] = 1.0;
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < M - N; ++i) {
            zc v = z[IDX2(i, j, M - N)];
            newmo[IDX2(N + i, j, M)] = (cmplxconj == 0) ? creal(v) : v;
        }
    const int total = nl * ny * npg;
    const int npts = omega_list ? n_omega : total;
    const size_t acc_scalar = (size_t)nci * nci, acc_mat = acc_scalar * MM;
    int nth = 1;
#ifdef _OPENMP
    nth = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    /* fewer points than threads: the points run one after another, each split over the threads */
    g_inner = (npts < nth) ? nth : 1;
    if (g_inner > 1) nth = 1;
    zc *th_h = calloc(acc_scalar * nth, sizeof(zc)), *th_s = calloc(acc_scalar * nth, sizeof(zc));
    zc *th_g = calloc(acc_mat * nth, sizeof(zc)), *th_r = calloc(acc_mat * nth, sizeof(zc));
    int status = 0;
    const int d = ncisp * ncipg;
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        scratch_t s;
        s.R = malloc(sizeof(zc) * MM); s.Rt = malloc(sizeof(zc) * MM); s.Rt2 = malloc(sizeof(zc) * MM);
        s.tmp = malloc(sizeof(zc) * MM); s.Mm = malloc(sizeof(zc) * N * N); s.Minv = malloc(sizeof(zc) * N * N);
        s.work = malloc(sizeof(zc) * N * N); s.piv = malloc(sizeof(int) * N);
        s.t2 = malloc(sizeof(zc) * 2 * (size_t)M * N);
        zc *rho[4], *gam = malloc(sizeof(zc) * MM), *g[4], *gtmp = malloc(sizeof(zc) * MM);
        for (int v = 0; v < 4; ++v) { rho[v] = malloc(sizeof(zc) * MM); g[v] = malloc(sizeof(zc) * MM); }
        zc *R = malloc(sizeof(zc) * MM);
        zc *hh = th_h + acc_scalar * tid, *ss = th_s + acc_scalar * tid;
        zc *gg = th_g + acc_mat * tid, *rr = th_r + acc_mat * tid;
#pragma omp for schedule(static)
        for (int t = 0; t < npts; ++t) {
            int w = omega_list ? omega_list[t] : t;
            int il = w / (ny * npg), iy = (w / npg) % ny, ipg = w % npg;
            /* Rtmp = R1(il) R2(iy) Rpg(ipg); R = Ref^H Rtmp Ref */
            zc *A = s.Rt, *Bm = s.Rt2, *Cm = s.tmp;
            for (int j = 0; j < M; ++j)
                for (int i = 0; i < M; ++i) {
                    A[IDX2(i, j, M)] = r1[(size_t)il + (size_t)nl * IDX2(i, j, M)];
                    Bm[IDX2(i, j, M)] = r2[(size_t)iy + (size_t)ny * IDX2(i, j, M)];
                }
            zgemm_cm(M, M, M, A, M, 0, Bm, M, Cm, M);
            for (int j = 0; j < M; ++j)
                for (int i = 0; i < M; ++i) Bm[IDX2(i, j, M)] = rpg[(size_t)ipg + (size_t)npg * IDX2(i, j, M)];
            zgemm_cm(M, M, M, Cm, M, 0, Bm, M, A, M);            /* A = Rtmp */
            zgemm_cm(M, M, M, A, M, 0, ref, M, Cm, M);           /* Rtmp Ref */
            zgemm_cm(M, M, M, ref, M, 2, Cm, M, R, M);           /* Ref^H Rtmp Ref */
            zc sv[4], hv[2];
            int nv = (cmplxconj == 2) ? 4 : 1;
            /* variants: 0 = RDM(R,MO), 1 = RDMConj(R,MO), 2 = RDM(R,conj MO), 3 = RDMConj(R,conj MO) */
            for (int v = 0; v < nv; ++v) {
                int cb = (v >= 2), ck = (v == 1) ? 1 : (v == 2 ? 1 : 0);
                if (v == 3) ck = 0; /* RDMConj(R, conj MO): ket conj(conj MO) = MO */
                if (rdm(M, N, R, newmo, cb, ck, &s, rho[v], &sv[v])) {
#pragma omp atomic write
                    status = 2;
                    continue;
                }
                make_gamma(&H, rho[v], gam, gtmp);
                if (v < 2) hv[v] = makeh(M, hone, gam, rho[v]) * sv[v];
                gradient(&H, gam, rho[v], sv[v], &s, g[v]);
            }
            if (status) continue;
            if (nv == 1) { hv[1] = hv[0]; }
            double wsp = weightsp[(size_t)il + (size_t)nl * iy];
            for (int ni = -qj; ni <= qj; ++ni)
                for (int nj = -qj; nj <= qj; ++nj) {
                    zc wig = (sp == 2) ? wignerfac(qj, ni, nj, roota[il], rootb[iy], rooty[il])
                                       : wignerfac(qj, ni, nj, roota[il], rootb[il], rooty[iy]);
                    for (int p = 0; p < ncipg; ++p)
                        for (int q = 0; q < ncipg; ++q) {
                            zc wv = weightpg[(size_t)ipg + (size_t)npg * ((size_t)p + (size_t)ncipg * q)] * wig;
                            int m = ni + qj + p * ncisp, n = nj + qj + q * ncisp;
                            /* (slot offset, variant) pairs of PHFTools.f90:149-162 */
                            int pairs = (cmplxconj == 2) ? 4 : 1;
                            static const int dm_[4] = {0, 0, 1, 1}, dn_[4] = {0, 1, 0, 1}, var_[4] = {0, 1, 3, 2};
                            for (int e = 0; e < pairs; ++e) {
                                int mm = m + dm_[e] * d, nn = n + dn_[e] * d, v = var_[e];
                                size_t so = (size_t)mm + (size_t)nci * nn;
                                zc sw = sv[v] * wsp;
                                if (e < 2) {
                                    hh[so] += hv[e] * wsp * wv;
                                    ss[so] += sw * wv;
                                }
                                zc *gd = gg + so, *rd = rr + so;
                                for (size_t ij = 0; ij < MM; ++ij) {
                                    gd[acc_scalar * ij] += g[v][ij] * wsp * wv;
                                    rd[acc_scalar * ij] += rho[v][ij] * sw * wv;
                                }
                            }
                        }
                }
        }
        free(s.R); free(s.Rt); free(s.Rt2); free(s.tmp); free(s.Mm); free(s.Minv); free(s.work); free(s.piv);
        free(s.t2); free(gam); free(gtmp); free(R);
        for (int v = 0; v < 4; ++v) { free(rho[v]); free(g[v]); }
    }
    /* reduce thread accumulators in thread order (deterministic) */
    memset(hmat, 0, sizeof(zc) * acc_scalar);
    memset(smat, 0, sizeof(zc) * acc_scalar);
    memset(gradmat, 0, sizeof(zc) * acc_mat);
    memset(rdmmat, 0, sizeof(zc) * acc_mat);
    for (int t = 0; t < nth; ++t) {
        for (size_t i = 0; i < acc_scalar; ++i) { hmat[i] += th_h[acc_scalar * t + i]; smat[i] += th_s[acc_scalar * t + i]; }
        for (size_t i = 0; i < acc_mat; ++i) { gradmat[i] += th_g[acc_mat * t + i]; rdmmat[i] += th_r[acc_mat * t + i]; }
    }
    if (cmplxconj == 2) { /* PHFTools.f90:174-179 */
        for (int a = 0; a < d; ++a)
            for (int b = 0; b < d; ++b) {
                hmat[(size_t)(d + a) + (size_t)nci * b] = conj(hmat[(size_t)b + (size_t)nci * (d + a)]);
                smat[(size_t)(d + a) + (size_t)nci * b] = conj(smat[(size_t)b + (size_t)nci * (d + a)]);
                hmat[(size_t)(d + a) + (size_t)nci * (d + b)] = hmat[(size_t)a + (size_t)nci * b];
                smat[(size_t)(d + a) + (size_t)nci * (d + b)] = smat[(size_t)a + (size_t)nci * b];
            }
    }
    free(th_h); free(th_s); free(th_g); free(th_r); free(newmo);
    g_inner = 1;
    return status;
}

int oracle_buildhsg(const zc *hone, const zc *htwo, const zc *bt, int nchol, const zc *ref, const zc *z,
                    const int *ngrid, int nci, int cmplxconj, int ncisp, int nocc, const zc *r1, const zc *r2,
                    const zc *rpg, const double *weightsp, const double *weightpg, const double *roota,
                    const double *rootb, const double *rooty, int qj, int sp, int npg, int ncipg, int nso,
                    const int *omega_list, int n_omega, int nthreads, zc *hmat, zc *smat, zc *gradmat,
                    zc *rdmmat)
{
    return oracle_buildhsg_ex(hone, htwo, bt, NULL, nchol, ref, z, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg,
                              weightsp, weightpg, roota, rootb, rooty, qj, sp, npg, ncipg, nso, omega_list, n_omega,
                              nthreads, hmat, smat, gradmat, rdmmat);
}

/* LocalG (PHFTools.f90:203-247) */
int oracle_localg(const zc *gradmat, const zc *rdmmat, const zc *smat, double e0_re, double e0_im, int nso, const zc *fsp, const zc *fpg,
                  const zc *fk, int nci, int ncisp, int ncipg, int cmplxconj, zc *G)
{
    const size_t MM = (size_t)nso * nso, ns = (size_t)nci * nci;
    const zc e0 = e0_re + I * e0_im;
    zc *rdm = calloc(MM, sizeof(zc));
    zc ovlp = 0;
    memset(G, 0, sizeof(zc) * MM);
    const int d = ncisp * ncipg;
    for (int ni = 0; ni < ncisp; ++ni)
        for (int nj = 0; nj < ncisp; ++nj)
            for (int p = 0; p < ncipg; ++p)
                for (int q = 0; q < ncipg; ++q) {
                    int m = ni + p * ncisp, n = nj + q * ncisp;
                    zc f = conj(fsp[ni]) * fsp[nj] * conj(fpg[p]) * fpg[q];
                    zc f00 = f * conj(fk[0]) * fk[0];
                    size_t s0 = (size_t)m + (size_t)nci * n;
                    for (size_t ij = 0; ij < MM; ++ij) {
                        G[ij] += f00 * gradmat[s0 + ns * ij];
                        rdm[ij] += f00 * rdmmat[s0 + ns * ij];
                    }
                    ovlp += f00 * smat[s0];
                    if (cmplxconj == 2) {
                        zc f11 = f * conj(fk[1]) * fk[1], f01 = f * conj(fk[0]) * fk[1], f10 = f * conj(fk[1]) * fk[0];
                        size_t s11 = (size_t)(m + d) + (size_t)nci * (n + d);
                        size_t s01 = (size_t)m + (size_t)nci * (n + d);
                        size_t s10 = (size_t)(m + d) + (size_t)nci * n;
                        for (size_t ij = 0; ij < MM; ++ij) {
                            G[ij] += f11 * conj(gradmat[s11 + ns * ij]) + f01 * gradmat[s01 + ns * ij] +
                                     f01 * conj(gradmat[s10 + ns * ij]);
                            rdm[ij] += f11 * conj(rdmmat[s11 + ns * ij]) + f01 * rdmmat[s01 + ns * ij] +
                                       f01 * conj(rdmmat[s10 + ns * ij]);
                        }
                        ovlp += f11 * smat[s11] + f01 * smat[s01] + f10 * smat[s10];
                    }
                }
    for (size_t ij = 0; ij < MM; ++ij) G[ij] = (G[ij] - e0 * rdm[ij]) / ovlp;
    free(rdm);
    return 0;
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
