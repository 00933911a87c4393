/*
 * phf_b200 -- C ABI of the B200 projected-HF grid kernel.
 *
 * Drop-in for the two routines of the reference's f2py module PHFTools_F (module phftools,
 * built by PHF_fort/makefile:7) that PHF.py calls for the projected energy and gradient:
 *
 *   phftools.buildhsg  -> phf_buildhsg       (PHF_fort/PHFTools.f90:10-201, called at PHF.py:44-45,70-71)
 *   phftools.localg    -> phf_localg         (PHF_fort/PHFTools.f90:203-247, called at PHF.py:76)
 *
 * Arrays use the reference's Fortran dummy-argument layouts (column-major), complex128 as
 * {re, im} pairs, so a binding passes f2py/numpy Fortran-ordered buffers unchanged:
 *   HOne(i,j)       = hone[i + M*j]                     M = nso spin orbitals
 *   HTwo(i,j,k,l)   = htwo[i + M*(j + M*(k + M*l))]     antisymmetrised <ij||kl>
 *   Ref(i,j)        = ref[i + M*j];   Z(a,i) = z[a + (M-nocc)*i]
 *   R1(il,i,j)      = r1[il + ngrid[0]*(i + M*j)];   R2(iy,i,j) = r2[iy + ngrid[1]*(i + M*j)]
 *   Rpg(ig,i,j)     = rpg[ig + npg*(i + M*j)]
 *   weightsp(il,iy) = weightsp[il + ngrid[0]*iy]
 *   weightpg(ig,p,q)= weightpg[ig + npg*(p + ncipg*q)]
 *   roota: ngrid[0] entries; rootb: ngrid[0] entries (ngrid[1] when sp == 2);
 *   rooty: ngrid[1] entries (ngrid[0] when sp == 2)
 *   Hmat(m,n)       = hmat[m + nci*n];   Gradmat(m,n,i,j) = gradmat[m + nci*(n + nci*(i + M*j))]
 *
 * Every entry point returns a status code instead of the reference's Fortran STOP.  All
 * computation runs on the current CUDA device; there is no CPU fallback: without a device
 * the calls return PHF_ERR_NO_DEVICE.
 */
#ifndef PHF_B200_H
#define PHF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double re, im;
} phf_complex;

enum phf_status {
    PHF_OK = 0,
    PHF_ERR_ARG = 1,            /* inconsistent sizes or arguments */
    PHF_ERR_SINGULAR = 2,       /* a rotated overlap C^H R C is exactly singular
                                   (reference: STOP "Error in ZGetRF", Wrappers.f90:311) */
    PHF_ERR_NOT_HERMITIAN = 3,  /* Hmat/Smat fail the check of PHFTools.f90:195-200
                                   (reference: STOP "Not Hermitian"); outputs are still written */
    PHF_ERR_NONFINITE = 4,      /* NaN/Inf in inputs or results */
    PHF_ERR_CUDA = 5,           /* CUDA runtime error */
    PHF_ERR_OOM = 6,            /* device allocation failed */
    PHF_ERR_UNSUPPORTED = 7,    /* size or option outside what this build implements */
    PHF_ERR_NO_DEVICE = 8       /* no CUDA device */
};

/* Arithmetic of the J/K contraction (the overlap inverse, determinants, weights and the
 * compensated grid sums are FP64 in every mode). */
enum phf_precision {
    PHF_PREC_FP64 = 0,      /* FP64 CUDA-core GEMMs (the plain FP64 form) */
    PHF_PREC_OZAKI_I8 = 1,  /* FP64-accurate emulation: int8 slices on tcgen05 tensor cores */
    PHF_PREC_BF16X3 = 2,    /* split-BF16 (hi + lo: ~16 significant bits), 3 products, FP32 accumulation (tcgen05) */
    PHF_PREC_TF32 = 3       /* TF32 (11 significant bits), FP32 accumulation (tcgen05) */
};

/* ---------------------------------------------------------------- drop-in entry points */

/* BuildHSG (PHF_fort/PHFTools.f90:10-48 declaration).  Dense HTwo in the Ref-MO basis, as
 * PHF.py passes it.  Host buffers in, host buffers out (outputs overwritten).
 * Returns PHF_ERR_NOT_HERMITIAN (outputs written) where the reference would STOP. */
int phf_buildhsg(const phf_complex *hone, const phf_complex *htwo, const phf_complex *ref, const phf_complex *z,
                 const int *ngrid, int npg, int nci, int cmplxconj, int ncisp, int ncipg, int nocc, int nso,
                 const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const double *weightsp,
                 const double *weightpg, const double *roota, const double *rootb, const double *rooty, int qj,
                 int sp, phf_complex *hmat, phf_complex *smat, phf_complex *gradmat, phf_complex *rdmmat);

/* BuildHSG with the two-electron integrals given as spatial Cholesky vectors in the
 * orthonormal AO basis: (pq|rs) = sum_L B_L(p,q) B_L(r,s), B_L(p,q) = bvec[p + n*(q + n*L)],
 * and the one-electron matrix h(p,q) = h[p + n*q] (n = nso/2).  Equivalent to phf_buildhsg with
 * HOne = Ref^H blockdiag(h,h) Ref and HTwo = the Ref-MO transform of the antisymmetrised
 * spin-orbital integrals (Main_PHF.py:22-33), without forming the n^4 tensor.
 * Requires Ref unitary (the reference's Ref is an orthonormal MO matrix). */
int phf_buildhsg_chol(const double *h, const double *bvec, int nchol, const phf_complex *ref, const phf_complex *z,
                      const int *ngrid, int npg, int nci, int cmplxconj, int ncisp, int ncipg, int nocc, int nso,
                      const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const double *weightsp,
                      const double *weightpg, const double *roota, const double *rootb, const double *rooty, int qj,
                      int sp, int precision, phf_complex *hmat, phf_complex *smat, phf_complex *gradmat,
                      phf_complex *rdmmat);

/* LocalG (PHF_fort/PHFTools.f90:203-247 declaration): G(M,M) = (sum f*f Gradmat - e0 sum f*f
 * Rdmmat) / sum f*f Smat.  fk has 1 entry (2 when cmplxconj == 2).  Host buffers. */
int phf_localg(const phf_complex *gradmat, const phf_complex *rdmmat, const phf_complex *smat, phf_complex e0,
               int nso, const phf_complex *fsp, const phf_complex *fpg, const phf_complex *fk, int nci, int ncisp,
               int ncipg, int cmplxconj, phf_complex *g);

/* BuildSC (PHF_fort/PHFTools.f90:464-537, with BuildSC_Vec of PHF_fort/BuildSC_dr.f90): the
 * grid-projected product of a coupled-cluster-shaped vector (c0, c1(M,M), c2(M,M,M,M), Fortran
 * layouts c1(a,b) = c1[a + M*b], c2(a,b,c,d) = c2[a + M*(b + M*(c + M*d))]) with the projection of the
 * reference determinant [I; 0], as LinDep.py:71-76 applies it: per grid point R = R1 R2 Rpg, the
 * transition density of [I; 0], c1 and c2 transformed with R^H, BuildSC_Vec, weighted by
 * weightsp det(R[:N,:N]) sum_pq weightpg conj(fpg_p) fpg_q (sum conj fsp)(sum fsp) and divided by the
 * projected overlap.  As in the reference's loop, rk, fk and the Wigner angles (roota, rootb, rooty,
 * qj) take no part (the Wigner factor is computed and then set to one, :516-518).  Host buffers in,
 * t0, t1(M,M), t2(M,M,M,M) out.  FP64 on the GPU; M^4 complex per tensor per grid point of device
 * memory, grid points run in chunks of a 4 GiB workspace. */
int phf_buildsc(phf_complex c0, const phf_complex *c1, const phf_complex *c2, int nocc, int nso, const int *ngrid,
                int npg, int qj, int ncisp, int ncipg, int ncik, const phf_complex *r1, const phf_complex *r2,
                const phf_complex *rpg, const phf_complex *rk, const double *roota, const double *rootb,
                const double *rooty, const double *weightsp, const double *weightpg, const phf_complex *fsp,
                const phf_complex *fpg, const phf_complex *fk, phf_complex *t0, phf_complex *t1, phf_complex *t2);

/* PbarHbarOlap (SUCCSD_Boson_cmplx/FPUCC.f90:14-48 declaration, body :49-272): the grid kernel of
 * projected CCSD, which the reference's PCC solver (Main.f90 PGCC -> BroydenIter, Broyden.f90) calls once
 * per iteration.  For every grid point (il, iy, ipg) with R = R1(il) R2(iy) Rpg(ipg), EvalKernel
 * (FPUCC.f90:529-602): the amplitudes (t1, t2) transformed by R (DSTT2: the Thouless form of R [1; T1]
 * and the double similarity transform of T2, FPUCC_Tools.f90:697-722, PCCCI.f90:14-276), the CCSD energy
 * and residuals of the transformed amplitudes with the Fock matrix of (hone, htwo) (CCRes.f90), and the
 * lambda / eps tensors of BuildKernSD (FPUCC_Tools.f90:291-436), summed with the weight
 * weightsp weightpg(ipg,p,q) Wigner(qj,m,n) conj(fsp(m)) fsp(n) conj(fpg(p)) fpg(q) over m, n, p, q; with
 * ncik == 2 a second pass with conjugated hone, htwo, t1, t2, R Rk(2) and weight times fk(2); with
 * sp == 2 the spin-flip components are projected out (ProjSz, MO order [occ alpha, occ beta, vir alpha,
 * vir beta]).  Layouts (Fortran, M = nso, v = nso - nocc):
 *   hone(i,j) = hone[i + M*j];  htwo(i,j,k,l) = htwo[i + M*(j + M*(k + M*l))]  antisymmetrised <ij||kl>
 *   t1(a,i) = t1[a + v*i];  t2(a,b,i,j) = t2[a + v*(b + v*(i + nocc*j))]      (a, b virtual from 0)
 *   r1, r2, rpg, weightsp, weightpg, roota, rootb, rooty as phf_buildhsg (npoints = ngrid);
 *   rk(t,i,j) = rk[t + ncik*(i + M*j)];  fsp: ncisp = 2*qj+1 entries, fpg: ncipg, fk: ncik
 *   outputs olap0, eolap0 (scalars), olapex1, eolapex1 (v x nocc), olapex2, eolapex2 (v,v,nocc,nocc).
 * ref and nao are accepted as in the reference (nao = nso/2 or 0) and not used.  trunode 1, 2 or -3 run
 * the SD kernel (BuildKernSD takes |trunode|); 3 also adds the (T) energy of the transformed amplitudes
 * to eps0 at every point (CCSD_T_Ene, SUCCSD_Boson_cmplx/CCSD_T.f90:10-108, FPUCC.f90:577-581; o^3 v^3
 * complex per point of extra device memory, a few points at a time); other values return PHF_ERR_ARG
 * (the reference STOPs).  FP64 on the GPU, nso <= 112; M^4 complex per grid point of device memory (grid
 * points run in chunks of `workspace` bytes, 0 = 16 GiB).  comm is not taken: the reference's rank
 * split over iy is a partial sum over grid points that callers add. */
int phf_pbarhbarolap(phf_complex *olap0, phf_complex *olapex1, phf_complex *olapex2, phf_complex *eolap0,
                     phf_complex *eolapex1, phf_complex *eolapex2, const phf_complex *hone, const phf_complex *htwo,
                     const phf_complex *ref, const phf_complex *t1, const phf_complex *t2, int nocc, int nao, int nso,
                     double enuc, int qj, int sp, const int *npoints, int npg, int ncisp, int ncipg, int ncik,
                     const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const phf_complex *rk,
                     const double *roota, const double *rootb, const double *rooty, const double *weightsp,
                     const double *weightpg, const phf_complex *fsp, const phf_complex *fpg, const phf_complex *fk,
                     int trunode, size_t workspace);

/* Device time in ms of the last phf_pbarhbarolap call's grid pipeline (from the first launch after the
 * inputs are uploaded to the end of the last sum, CUDA events on its stream) and the FP64 flops its
 * GEMMs executed (8 m n k per complex product).  No counterpart in the reference. */
int phf_pbarhbarolap_stats(double *device_ms, double *gemm_flops);

/* ---------------------------------------------------------------- plan API
 * A plan holds the Hamiltonian, the grid and the device workspace, so that repeated
 * energy/gradient evaluations (one per optimiser step, PHF.py:55-91) upload only Z or C. */
typedef struct phf_plan phf_plan;

typedef struct {
    int nso, nocc;
    int nchol;                                /* > 0: Cholesky form (h, bvec); 0: dense (hone, htwo) */
    const double *h, *bvec;                   /* Cholesky form, layouts as phf_buildhsg_chol */
    const phf_complex *hone, *htwo;           /* dense form, layouts as phf_buildhsg */
    const phf_complex *ref;                   /* Ref(M,M) */
    const int *ngrid;
    int npg, nci, ncisp, ncipg, cmplxconj, qj, sp;
    const phf_complex *r1, *r2, *rpg;
    const double *weightsp, *weightpg, *roota, *rootb, *rooty;
    int precision;                            /* enum phf_precision */
    int slices;                               /* int8 slices per operand for PHF_PREC_OZAKI_I8 (0 = default) */
    size_t workspace_bytes;                   /* per-chunk workspace budget (0 = default: 6 GiB, or 45 % of
                                                 the free device memory for jk_form 3 when that is more) */
    int jk_form;                              /* Cholesky form only: 0 = automatic, 1 = exchange through the
                                                 spatial ERI matrix (n^2 x n^2, built once per plan and kept),
                                                 2 = factorized (rank-N, no n^4 tensor, FP64 only),
                                                 3 = streamed: the exchange rows regenerated from the Cholesky
                                                 vectors panel by panel in every chunk, each panel used
                                                 against the whole chunk (no n^4 tensor; memory of one panel);
                                                 automatic picks 1 for n <= 128, else 3 */
    int gradient_mode;                        /* phf_plan_eval_device only: 0 = the reference's gradient
                                                 (bra-side derivative, Gradient/LocalG of PHFTools.f90);
                                                 1 = exact dE/dC* of E = Re H/|Re S|, adding the ket-side
                                                 term (spatial-ERI form, nci == 1) */
    int fp64_library_gemm;                    /* PHF_PREC_FP64, spatial-ERI form: 1 = run the exchange GEMM
                                                 with cuBLAS DGEMM instead of this library's FP64 kernel
                                                 (a library-tuned FP64 comparison form) */
    int point_begin, point_end;               /* evaluate only grid points [point_begin, point_end) of the
                                                 flattened order (il*ngrid[1] + iy)*npg + ipg; 0, 0 = all.
                                                 Partial sums over disjoint ranges add up to the full sums
                                                 (the rank split of PHFTools.f90:53-57) */
    int exchange_panel;                       /* jk_form 3: spatial indices i per exchange panel (rows (i, k)
                                                 of the exchange matrix formed at once); 0 = automatic
                                                 (at most 8192 rows, fewest padded rows).  With the
                                                 exchange symmetry, a panel starting at i0 takes
                                                 max(1, exchange_panel n / (n - i0)) indices, so that each
                                                 panel's Gram block stays within exchange_panel n x n^2 */
    int autotune;                             /* 1: at the plan's first evaluation, time the candidate launch
                                                 choices of every GEMM shape the plan uses (FP64 GEMM tile
                                                 shape, int8 GEMM raster group) and keep the fastest; the table
                                                 is shared by all plans of the process.  Results are bitwise
                                                 those of the untuned plan */
    int exchange_symmetry;                    /* jk_form 3: 0 = automatic (on where available), 1 = on, 2 = off.
                                                 On: the exchange uses K(rho^T) = K(rho)^T of real integrals --
                                                 rows (i <= k) against the symmetric half of each density and
                                                 rows (i < k) against the antisymmetric half, half the exchange
                                                 GEMM's work and of its rows' regeneration; the FP64 form and the
                                                 tensor-core forms with n > 64 (n <= 64 tensor-core plans slice
                                                 the densities in the fused kernel and run the full rows) */
} phf_plan_desc;

int phf_plan_create(const phf_plan_desc *desc, phf_plan **plan);
int phf_plan_destroy(phf_plan *plan);

/* buildhsg semantics for a new Z with the plan's Hamiltonian, grid and Ref (host buffers). */
int phf_plan_buildhsg(phf_plan *plan, const phf_complex *z, phf_complex *hmat, phf_complex *smat,
                      phf_complex *gradmat, phf_complex *rdmmat);

/* Device-resident evaluation for a determinant C (device, M x N row-major, [alpha; beta]
 * spin-orbital order, in the basis of the plan's Hamiltonian: AO for the Cholesky form).
 * Writes, in device memory on `stream` (a cudaStream_t, 0 = legacy default stream):
 *   d_hs[2*a], d_hs[2*a+1]   -- sum_w W_a(w) N_w h_w and sum_w W_a(w) N_w for slot a = m + nci*n
 *   d_yg[a*M*N + r*N + j]    -- sum_w W_a(w) N_w [(1 - rho_w) F_w X_w + h_w X_w]
 *   d_yr[a*M*N + r*N + j]    -- sum_w W_a(w) N_w X_w,   X_w = R_w C (C^H R_w C)^-1
 * so that Gradmat_a = Yg_a C^H, Rdmmat_a = Yr_a C^H, and for nci == 1 the energy is
 * E = Re H / |Re S| and the reference's gradient is (Yg - E Yr) / S.  With gradient_mode 1 the
 * outputs are the symmetrised sums Yg = (Yg_bra + Yg_ket)/2, Yr = (Yr_bra + Yr_ket)/2, where
 * Yg_ket = sum_w conj(W_a(w) N_w) R_w^H [(H1 + Gamma_w^H) C - C W_w^H + conj(h_w) C] S_w^-H and
 * Yr_ket = sum_w conj(W_a(w) N_w) R_w^H C S_w^-H, and dE/dC* = (Yg - E sgn(Re S) Yr) / |Re S|
 * exactly.  cmplxconj must be 0 or 1. */
int phf_plan_eval_device(phf_plan *plan, const phf_complex *d_c, phf_complex *d_hs, phf_complex *d_yg,
                         phf_complex *d_yr, void *stream);

/* phf_plan_eval_device without its synchronisation, for device-resident loops (one optimiser step
 * per host round trip): the evaluation is queued on `stream` and returns at once; the two status
 * words -- d_status[0]: bit 0 a rotated overlap was exactly singular, bit 1 non-finite; d_status[1]:
 * tensor-core pipeline error code (0 = none) -- are copied to device memory on the same stream, to
 * be read by the caller with its own results (PHF_ERR_SINGULAR / PHF_ERR_NONFINITE / PHF_ERR_CUDA
 * where phf_plan_eval_device would return them).  Returns only errors found while queueing.  The
 * plan's buffers are in use until the stream reaches the end of the evaluation: do not queue a
 * second evaluation of the same plan on another stream before then.  No counterpart in the
 * reference (its driver synchronises every call). */
int phf_plan_eval_device_async(phf_plan *plan, const phf_complex *d_c, phf_complex *d_hs, phf_complex *d_yg,
                               phf_complex *d_yr, int *d_status, void *stream);

/* Batched evaluation of independent instances (the many-instance workload of uneven orbital
 * counts): plans[i] evaluates determinant d_c[i] into d_hs[i], d_yg[i], d_yr[i] exactly as
 * phf_plan_eval_device.  All instances run as one CUDA graph on `stream`, captured on first use
 * for this set of plans and buffers (again after any plan is destroyed or a buffer changes) with
 * the instances spread over 4, 8 or 16 concurrent branches -- the count that timed fastest when the
 * set was captured.  Synchronous; returns the first failing instance's status.  No counterpart in
 * the reference (its driver runs one PHF instance at a time). */
int phf_eval_batch(phf_plan *const *plans, int count, const phf_complex *const *d_c, phf_complex *const *d_hs,
                   phf_complex *const *d_yg, phf_complex *const *d_yr, void *stream);
/* Concurrent branches of the batch graph phf_eval_batch captured last (0 before any). */
int phf_batch_branches(void);

/* Grid points per pipeline chunk chosen by the plan, and its device workspace in bytes. */
int phf_plan_info(const phf_plan *plan, int *chunk, size_t *workspace_bytes);

/* FP64-accurate real GEMM on the int8 tensor cores (the arithmetic of PHF_PREC_OZAKI_I8):
 * D (m x n, row-major, ldd) = A (m x k, row-major, lda) * B, with B given transposed as
 * Bt (n x k, row-major, ldb).  `slices` int8 slices per operand (1..7; balanced base-254 digits,
 * each ~8 bits; the error of an entry is below (slices+1) k 2^(-7 slices) max|A_i.| max|B_.j|, and in
 * practice near 254^(-slices) sqrt(k) max|A_i.| max|B_.j|).  Device pointers; synchronous on `stream`.
 * No counterpart in the reference (its J/K is a dense FP64 loop, PHFTools.f90:310-337). */
int phf_ozaki_dgemm(int m, int n, int k, int slices, const double *dA, long long lda, const double *dBt,
                    long long ldb, double *dD, long long ldd, void *stream);

/* The real GEMM of phf_ozaki_dgemm in each tensor-core precision that plans offer for their J/K
 * contractions, with the same arithmetic: PHF_PREC_OZAKI_I8 with `slices` int8 slices
 * (0 = 5); PHF_PREC_BF16X3: each row of A and column of B scaled by a power of two, split into
 * BF16 high and low parts (about 16 significant bits), hi*hi + hi*lo + lo*hi on the tensor cores;
 * PHF_PREC_TF32: TF32 operands (10 fraction bits, round to nearest).  Both accumulate in FP32 over
 * segments of 512 k-elements whose results are summed in FP64 (the tensor core's FP32 sums round
 * towards zero, which over long same-sign sums is the dominant error).  `slices`
 * is ignored for the floating-point precisions; PHF_PREC_FP64 is PHF_ERR_ARG.  Device pointers;
 * synchronous on `stream`.  No counterpart in the reference. */
int phf_tc_dgemm(int m, int n, int k, int precision, int slices, const double *dA, long long lda, const double *dBt,
                 long long ldb, double *dD, long long ldd, void *stream);

/* Inverse, determinant and log-determinant of `batch` complex n x n matrices (interleaved re/im
 * doubles, row-major, matrix b at dS + 2 n^2 b), the step inside every grid point of BuildHSG: it
 * replaces InvertC (ZGETRF + ZGETRI) and determinantC (ZGETRF), PHF_fort/Wrappers.f90:195-336, as
 * RDM calls them (PHF_fort/PHFTools.f90:259-260).  FP64 Gauss-Jordan elimination with partial
 * pivoting on |re| + |im| (the pivots of LU with partial pivoting), n <= 112.  dSinv as dS; ddet and
 * dlogdet hold one complex each per matrix (log det = log|det| + i arg, arg in (-pi, pi]); dflag is
 * one device int the call overwrites.  A singular matrix returns PHF_ERR_SINGULAR and a non-finite
 * entry PHF_ERR_NONFINITE, with that matrix's outputs zeroed (det 0, log det -inf).  Device
 * pointers; synchronous on `stream`. */
int phf_overlap_inverse(int n, int batch, const double *dS, double *dSinv, double *ddet, double *dlogdet, int *dflag,
                        void *stream);

/* The same product as phf_ozaki_dgemm for callers that cannot allocate device memory at the
 * point of the call: programs whose device memory belongs to another allocator (a framework's
 * caching pool, or a fixed arena reserved at start-up, where a cudaMalloc of this library's own
 * would fail or split the pool), and loops that must never enter the driver's allocator (cudaMalloc
 * and cudaFree can synchronize the device).  No counterpart in the reference.  Scratch (int8
 * slices, exponents, error flag) lives in one static device array of 32 MiB that every GPU loading
 * this library holds until exit; sizes needing more (see phf_ozaki_dgemm_noalloc_scratch_bytes)
 * return PHF_ERR_UNSUPPORTED.  No cudaMalloc/cudaFree or allocating library call is made.  All
 * calls share the array and it keeps the last call's contents (the parts that must start at zero
 * are cleared on each call): calls that overlap on the GPU race.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress, with that device current); make that first
 * call before any stream capture.  Synchronous on `stream`; a failed synchronisation is reported
 * as PHF_ERR_CUDA with the message "stream synchronize failed", as for phf_ozaki_dgemm. */
int phf_ozaki_dgemm_noalloc(int m, int n, int k, int slices, const double *dA, long long lda, const double *dBt,
                            long long ldb, double *dD, long long ldd, void *stream);
/* Scratch bytes phf_ozaki_dgemm_noalloc needs for these sizes; 0 for arguments it rejects
 * (m, n or k below 1, slices outside 1..7). */
size_t phf_ozaki_dgemm_noalloc_scratch_bytes(int m, int n, int k, int slices);

/* ---------------------------------------------------------------- diagnostics */
const char *phf_status_string(int status);
/* Message of the last failing call on this thread ("" when none). */
const char *phf_last_error(void);
/* Number of kernels this library has launched in this process. */
unsigned long long phf_kernel_launches(void);
/* Per-kernel-class timing with CUDA events on the launching stream, for roofline reports:
 * class 0 = J/K contraction GEMMs, 1 = other GEMMs, 2 = overlap inverse, 3 = memory-bound
 * kernels.  Enabling clears earlier records; read returns the summed device time of the
 * launches recorded since (it waits for their end events). */
int phf_profile_enable(int on);
int phf_profile_read(int kernel_class, double *total_ms, unsigned long long *launches);
/* GEMM shapes the launch tuner has timed so far in this process (plans created with autotune). */
int phf_tuned_shapes(void);
/* Whether the int8 GEMM (1 to 5 slices) issues one tensor-core MMA per A slice against the B slices
   it multiplies, laid side by side (default 1), or one MMA per slice pair (0).  The int32 sums are the
   same, so results are identical either way; the setting exists for comparisons.  Returns the previous
   setting.  Plans captured into CUDA graphs keep the form they were captured with. */
int phf_int8_wide_mma(int on);
/* Plans created while this is 1 (the default) and that form their densities on the int8 path (int8
   slices, n > 64) also form the per-point product F X = (H1 + J - K) X there: one batched int8 GEMM
   over the chunk's points (X's columns and F's rows as slices, k = 2M) instead of an FP64 GEMM per
   point; 0 keeps the FP64 product; a value above 1 also caps the points per sub-batch of that GEMM
   (otherwise sized to 1 GiB of slices).  Returns the previous setting.  No counterpart in the reference. */
int phf_int8_fock_product(int on);
/* Library version string. */
const char *phf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PHF_B200_H */
