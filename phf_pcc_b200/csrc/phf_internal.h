// Internal interfaces between the translation units of the library.
#pragma once
#include <algorithm>
#include <complex>
#include <functional>
#include <string>
#include <vector>

#include "phf_common.cuh"

namespace phf {

using cd = std::complex<double>;

// Device allocations owned by a plan, freed together.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct Arena {
    std::vector<DevBuf> bufs;
    size_t total = 0;
    ~Arena() { release(); }
    void release() {
        for (auto &b : bufs)
            if (b.p) cudaFree(b.p);
        bufs.clear();
        total = 0;
    }
    // frees one buffer of this arena early (no-op for a pointer it does not own)
    void free_one(void *ptr) {
        for (auto it = bufs.begin(); it != bufs.end(); ++it)
            if (it->p == ptr) {
                cudaFree(it->p);
                total -= it->bytes;
                bufs.erase(it);
                return;
            }
    }
    template <typename T>
    int alloc(T **out, size_t count) {
        size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(PHF_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
            return PHF_ERR_OOM;
        }
        bufs.push_back({p, bytes});
        total += bytes;
        *out = reinterpret_cast<T *>(p);
        return PHF_OK;
    }
};


// Per-shape launch choices found by timing (plans created with autotune): the FP64 GEMM's tile
// shape and the int8 GEMM's raster group.  Every candidate of a shape computes bitwise the same
// result (same per-element summation order), so a choice changes only the time.
struct TuneKey {
    int kind;                 // 0: FP64 GEMM tile shape, 1: int8 GEMM raster group
    long long a, b, c, d, e;  // shape and layout parameters of the launch
    bool operator==(const TuneKey &o) const {
        return kind == o.kind && a == o.a && b == o.b && c == o.c && d == o.d && e == o.e;
    }
};
struct TuneCall {
    TuneKey key;
    std::vector<int> candidates;
    std::function<int(int, cudaStream_t)> launch;  // launch with a candidate on a stream
};
// the table: -1 when the shape has not been tuned
int tuned_choice(const TuneKey &key);
int tuned_entries();
// non-zero: the int8 GEMM issues one MMA per slice pair instead of the wide issue (same results),
// for comparisons
extern int g_narrow_mma;
extern int g_fx_i8;  // plans created while > 0 form F X on the int8 path where they use int8 densities (default 1;
                     // a value above 1 caps the points per sub-batch)
// while non-null, the GEMM launchers append every launch they make (thread-local)
extern thread_local std::vector<TuneCall> *t_tune_record;
// times every candidate of every recorded launch whose shape is not in the table yet, keeps the fastest
int tune_recorded(std::vector<TuneCall> &calls, cudaStream_t st);

// Largest N (occupied orbitals) whose N x N overlap fits the shared-memory inverse.
constexpr int kMaxOverlapN = 112;


// overlap_inverse.cu
size_t overlap_inverse_smem(int N);
int overlap_inverse(int N, int batch, const zc *S, long long s_rs, long long s_bs, zc *Sinv, long long i_rs,
                    long long i_bs, zc *det, zc *logdet, int *flag, cudaStream_t st);

// phf_kernels.cu
int launch_tprime(int Ltot, int N, int b, zc *T, long long ldT, zc *e2part, cudaStream_t st);
int launch_rowsum(int nrows, int ncols, const zc *in, zc *out, double scale, cudaStream_t st);
// out[w] = scale tr(C^H X_w) (minus sub_scale sub[w] with `sub`); with `add`, X_w <- X_w + add_w
// afterwards (same layout as X)
int launch_trace_conj(int M, int N, int b, const zc *C, zc *X, long long ldX, zc *out, double scale,
                      cudaStream_t st, const zc *add = nullptr, const zc *sub = nullptr, double sub_scale = 0.0);
int launch_add_inplace(int M, int N, int b, const zc *A, zc *G, long long ldX, cudaStream_t st);
// Gamma's diagonal spin blocks += J (+ h, the one-electron matrix, when given)
int launch_add_coulomb_diag(int n, int b, const double *Jr, long long jrs, long long jcs, zc *Gam, cudaStream_t st,
                            const double *h = nullptr);
int launch_spin_block_y(int n, int N, int bc, int w0, int blk, const zc *R1b, const zc *T2, long long ld2, zc *Ys,
                        long long ld, cudaStream_t st);
int launch_epilogue(int M, int N, int b, zc *G, zc *X, long long ldX, const zc *det, const zc *e1,
                    const zc *e2, zc *scal, cudaStream_t st);
size_t accumulate_scratch_bytes(int nslot, int M, int N, int b);
int launch_accumulate(int nslot, int M, int N, int b, const zc *Wt, long long nomega, long long w0, const int *slotmap,
                      const zc *G, const zc *R, long long ldX, const zc *scal, zc *accG, zc *compG, zc *accR,
                      zc *compR, zc *accHS, zc *compHS, void *scratch, cudaStream_t st, int conj_weights = 0);
int launch_fold_comp(long long n, zc *a, const zc *c, cudaStream_t st);
int launch_ket_prep(int M, int N, int b, const zc *Hb, const zc *bra, const zc *e1, const zc *e2, zc *V, long long ld,
                    cudaStream_t st);
int launch_scale_conj_det(int M, int N, int b, const zc *det, zc *P, long long ld, cudaStream_t st);
int launch_average(long long n, const zc *a, const zc *b, zc *out, cudaStream_t st);
int launch_permute_h2(int M, const zc *H2, zc *H2r, cudaStream_t st);
int launch_permute_rows(int M, int N, int nbatch, const int *rowmap, const zc *in, long long ldin, long long bs_in,
                        zc *out, long long bs_out, cudaStream_t st);
int launch_localg(int MM, int nterm, const zc *coef_g, const zc *coef_r, const long long *slot_of_term,
                  const int *conj_of_term, const zc *gradmat, const zc *rdmmat, long long nslot, zc e0, zc ovlp, zc *G,
                  cudaStream_t st);

int launch_gather_p(int n, int b, const zc *rho, zc *P, long long ldp, cudaStream_t st);
int launch_gather_kin(int n, int b, const zc *rho, zc *Kin, long long ldk, cudaStream_t st);
// streamed FP64 form: EKp[(i - i0) n + k][l n + j] = G[(i - i0) n + l][k n + j] for one panel of ipanel i's
int launch_ek_panel(int n, int ipanel, const double *G, long long ldg, double *EKp, long long lde, cudaStream_t st);
// The bra's real operand for rho = X bra^H as a real GEMM on interleaved (re, im) rows of X: row 2j =
// (Re b_j0, Im b_j0, Re b_j1, ...), row 2j + 1 = (-Im b_j0, Re b_j0, ...) (bra M x N row-major).
int launch_bra_rho_operand(int M, int N, const zc *bra, double *out, cudaStream_t st);
int launch_assemble_gamma(int n, int b, const zc *J, long long ldj, const double *Jr, long long jrs, long long jcs,
                          const zc *Kc, long long ldk, const double *Kr, long long krs, long long kcs, zc *Gam,
                          cudaStream_t st, int ksym = 0, const double *h = nullptr);
// symmetric exchange form, FP64: the panel's symmetric rows EKs (rows_s x n(n+1)/2) and antisymmetric
// rows EKa (x n(n-1)/2) from its Gram block (as oz_slice_ek_sym_panel), and Kin's symmetric rows (pair_le
// order) followed by its antisymmetric rows (pair_lt order) from the dense densities
int launch_ek_sym_panel(int n, int i0, int ipanel, int k0, const int *pairs, const double *G, long long ldg,
                        double *EKs, double *EKa, cudaStream_t st);
int launch_gather_kin_sym(int n, int b, const int *pairs, const zc *rho, zc *Kin, long long ldk, cudaStream_t st);

// ozaki_i8.cu: FP64-accurate GEMM from int8 slices on tcgen05.  The slice-count argument S is 1..7
// int8 slices, or one of two floating-point operand formats contracted by the same kernel:
constexpr int OZ_FMT_BF16X3 = 8;  // BF16 high + low parts, hi*hi + hi*lo + lo*hi, FP32 accumulation
constexpr int OZ_FMT_TF32 = 9;    // TF32 values, FP32 accumulation
bool oz_format_ok(int S);
int oz_slots(int S);  // bytes per operand element in the slice buffers
long long oz_pad_rows(long long m);
long long oz_pad_cols(long long n);
long long oz_pad_k(long long k);
size_t oz_slice_bytes(long long rows_pad, long long k, int S);  // bytes of an operand's int8 slices
// ERI form, n <= 64: density columns of the K and P operands sliced straight from X and bra
bool oz_rho_slice_ok(int n);
int oz_rho_slice(int n, int N, int bc, const zc *Xs, long long ld, const zc *bra, int S, signed char *Ksl, int *eK,
                 signed char *Psl, int *eP, cudaStream_t st);
int oz_slice_rows(int m, int k, const double *A, long long lda, int S, long long rows_pad, signed char *out, int *ea,
                  cudaStream_t st);
int oz_slice_rows_strided(int m, int k, const double *A, long long lda, long long cs, int S, long long rows_pad,
                          signed char *out, int *ea, cudaStream_t st);
// Exchange columns (8 per point) and Coulomb columns (2 per point) of points 0 .. bc-1 of the densities
// rho_w (element [r][q] of point w at rho[w ws + r rs + q]; rs, ws even), sliced with their exponents.
int oz_slice_density(int n, int bc, const zc *rho, long long rs, long long ws, int S, signed char *Ksl, int *eK,
                     long long npadK, signed char *Psl, int *eP, long long npadP, cudaStream_t st);
int oz_gemm_t(int m, int n, int k, int S, const signed char *Asl, const int *ea, const signed char *Bsl, const int *eb,
              double *D, long long ldd, int accumulate, int trans, int *err, cudaStream_t st,
              int gamma_n = 0);  // gamma_n > 0: -K^T written into Gamma (exchange GEMM, m = n^2)
// Optional operand ranges and exchange-to-Gamma row modes of oz_gemm_ex:
//   b_rows_pad, b_row0: B rows (the output's columns) [b_row0, b_row0 + n) of a slice buffer of
//     b_rows_pad rows (0: a buffer of oz_pad_cols(n) rows), eb indexed by that buffer's rows;
//   gamma_mode: Gamma output rows 0 = exchange rows i n + k; 1 = symmetric pairs (i <= k), 2 =
//     antisymmetric pairs (i < k), pair of global row g = g_pairs[g] (i << 16 | k).
struct OzEx {
    long long b_rows_pad = 0;
    int b_row0 = 0;
    int gamma_mode = 0;
    const int *g_pairs = nullptr;
};
// oz_gemm_t with A rows [a_row0, a_row0 + m) of a slice buffer of a_rows_pad rows (ea indexed by that
// buffer's rows) and, in the Gamma mode, output row 0 at exchange row g_row0 (a panel of the exchange rows)
// Batched F_w X_w (F M x M, X M x N complex, one product per grid point w of `batch`) on the int8 path: A =
// oz_slice_xcols rows (w N + j), B = oz_slice_fock_rows rows (w 2M + 2c + part), k = 2M; the result lands
// at GX + c ld + w N + j (complex), GX's rows ld apart.  Single-pass int8 slice counts only.
int oz_gemm_fx(int M, int N, int batch, int S, const signed char *Asl, long long a_rows_pad, const int *ea,
               const signed char *Bsl, long long b_rows_pad, const int *eb, zc *GX, long long ld, int *err,
               cudaStream_t st);
// whether oz_gemm_fx takes M and S (single-pass int8 slices, k = 2M within one exact pass)
bool oz_fx_ok(int M, int S);
// slices of F_w's rows for oz_gemm_fx (F_w at F + w fs, rows of M complex): 2 batch M rows, k = 2M
int oz_slice_fock_rows(int M, int batch, const zc *F, long long fs, int S, long long rows_pad, signed char *out,
                       int *eb, cudaStream_t st);
// slices of X_w's columns for oz_gemm_fx (X_w[i][j] at X + i ld + w N + j): batch N rows, k = 2M
int oz_slice_xcols(int M, int N, int batch, const zc *X, long long ld, int S, long long rows_pad, signed char *out,
                   int *ea, cudaStream_t st);
int oz_gemm_ex(int m, int n, int k, int S, const signed char *Asl, long long a_rows_pad, int a_row0, const int *ea,
               const signed char *Bsl, const int *eb, double *D, long long ldd, int accumulate, int trans, int *err,
               cudaStream_t st, int gamma_n, int g_row0, const OzEx &ex = OzEx());
// slices of the exchange rows (i, k), i in [i0, i0 + ipanel), from the panel's Gram block G
// (G[(i - i0) n + l][k n + j] = sum_L B_L[i][l] B_L[k][j], row stride ldg); k-index l n + j
int oz_slice_ek_panel(int n, int ipanel, const double *G, long long ldg, int S, long long rows_pad, signed char *out,
                      int *ea, cudaStream_t st);
// Symmetric exchange form (n <= 65535; pairs tables: pair t -> i << 16 | k in row order, i <= k):
// the symmetric rows (pairs (i, k), i in [i0, i0 + ipanel), k >= i; rows_s = sum (n - i)) and the
// antisymmetric rows (k > i; rows_s - ipanel) of one panel, sliced from its Gram block
// G[(i - i0) n + l][(k - k0) n + j] (row stride ldg >= (n - k0) n, k0 <= i0)
int oz_slice_ek_sym_panel(int n, int i0, int ipanel, int k0, const int *pairs, const double *G, long long ldg, int S,
                          long long rows_pad_s, signed char *out_s, int *e_s, long long rows_pad_a, signed char *out_a,
                          int *e_a, cudaStream_t st);
// the symmetric and antisymmetric exchange columns (8 each per point) and the symmetric Coulomb columns
// (2 per point) of the densities, k-indices in pair order (see ozaki_i8.cu)
int oz_slice_density_sym(int n, int bc, const int *pairs, const zc *rho, long long rs, long long ws, int S,
                         signed char *Ks, int *eKs, signed char *Ka, int *eKa, long long npadK, signed char *Psl,
                         int *eP, long long npadP, cudaStream_t st);
// out (L x n(n+1)/2, FP64): B_L[l][j] (2 - delta_lj) at k-index pair_le(l, j), the Cholesky operand of the
// symmetric Coulomb contraction
int oz_cholesky_pairs(int n, int L, const double *Bst, const int *pairs, double *out, cudaStream_t st);
int oz_gemm_splitk(int m, int n, int k, int S, const signed char *Asl, const int *ea, const signed char *Bsl,
                   const int *eb, double *D, long long ldd, int trans, int nsplit, double *part, int *err,
                   cudaStream_t st);
int oz_gemm(int m, int n, int k, int S, const signed char *Asl, const int *ea, const signed char *Bsl, const int *eb,
            double *D, long long ldd, int accumulate, int *err, cudaStream_t st);

// Everything a plan owns: sizes, grid tables, Hamiltonian and the chunk workspace.
struct PlanImpl {
    int device = 0;
    bool chol = false;
    int n = 0, M = 0, N = 0, L = 0;
    int prec = PHF_PREC_FP64, slices = 0;
    int eri = 0;                     // exchange via the spatial ERI matrix (1) or factorized Cholesky (0)
    int streamed = 0;                // ERI form without the stored n^4 matrix: its rows are regenerated
                                     // from the Cholesky vectors in panels of ek_ipanel spatial indices i,
                                     // each used against the whole chunk and then overwritten
    int ek_ipanel = 0, ek_npanel = 0;
    int ek_sym = 0;                  // streamed form with the exchange symmetry (pairs i <= k, i < k)
    std::vector<int> ek_i0;          // symmetric form: panel p covers indices [ek_i0[p], ek_i0[p + 1])
    int *pairs_le = nullptr, *pairs_lt = nullptr;  // pair t -> i << 16 | k, i <= k, resp. i < k, row order
    int *eb_a = nullptr;             // exponents of the antisymmetric density columns (tensor-core form)
    size_t bsl_a_off = 0;            // byte offset of their slices in Bsl
    int exact = 0;                   // also accumulate the ket-side gradient (gradient_mode 1)
    int library_gemm = 0;            // FP64 exchange GEMM through cuBLAS (comparison form)
    void *cublas = nullptr;          // cublasHandle_t when library_gemm
    // CUDA graphs of the launch sequences replayed per call (key 0..3: variant of buildhsg, 4: the
    // whole eval_device pass), captured on first use on a private stream
    cudaStream_t cap_stream = nullptr;
    cudaStream_t side = nullptr;             // second stream: the Coulomb GEMMs beside the exchange GEMM
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t gexec[5] = {};
    unsigned long long glaunch[5] = {};  // kernels in each graph (for the launch counter)
    bool graphs_ok = true;
    bool autotune = false, tuned = false;    // time the launch choices of this plan's shapes once
    int nl = 0, ny = 0, npg = 0, nomega = 0;
    int wbeg = 0, wend = 0;          // grid points evaluated: [wbeg, wend)
    int nci = 0, ncisp = 0, ncipg = 0, cmplxconj = 1, qj = 0, sp = 1, nb = 0;
    std::vector<int> perm;           // working index -> reference index
    std::vector<cd> ref_host;        // Ref row-major (reference order)

    Arena arena;
    // persistent device data
    zc *R1 = nullptr, *R2 = nullptr, *Rpg = nullptr;  // working order, row-major
    zc *R1b = nullptr;  // Cholesky forms: R1's 2 x 2 spin blocks when R1 has no other nonzeros (nl x n x 4)
    zc *Refw = nullptr;                                // Ref with rows in working order, row-major
    zc *Wt = nullptr;                                  // nb^2 x nomega
    long long *offs = nullptr;                         // 3 * nomega
    int *slotmap = nullptr;                            // 4 x nb^2
    int *permdev = nullptr;                            // 2M: [0,M) working->reference, [M,2M) reference->working
    double *h = nullptr, *Bst = nullptr;               // Cholesky form
    bool fold_h = false;  // exchange-matrix forms with an exactly symmetric h: Gamma holds H1 + J - K
    zc *H1 = nullptr, *H2r = nullptr;                  // dense form
    // per evaluation
    zc *bra = nullptr, *ket = nullptr, *kety = nullptr, *newmo = nullptr, *newmoc = nullptr;
    zc *T1 = nullptr, *T2 = nullptr, *V = nullptr;
    // chunk workspace
    int b = 0;
    zc *Ys = nullptr, *Ys2 = nullptr, *S = nullptr, *Sinv = nullptr, *Xs = nullptr, *HX = nullptr, *GX = nullptr,
       *W = nullptr, *T = nullptr, *Q = nullptr, *Pv = nullptr, *Gv = nullptr, *det = nullptr, *logdet = nullptr,
       *e1 = nullptr, *e2 = nullptr, *e2part = nullptr, *scal = nullptr;
    int *flag = nullptr;
    // accumulators
    zc *accG = nullptr, *compG = nullptr, *accR = nullptr, *compR = nullptr, *accHS = nullptr, *compHS = nullptr;
    zc *tmpG = nullptr, *outMM = nullptr;
    void *acc_scratch = nullptr;       // partial sums of the two-stage accumulation
    // ket-side gradient (exact mode)
    zc *Hb = nullptr, *Vk = nullptr, *Pk = nullptr, *Pk2 = nullptr, *Prk = nullptr, *Prk2 = nullptr;
    zc *accKG = nullptr, *compKG = nullptr, *accKR = nullptr, *compKR = nullptr, *dummyHS = nullptr;
    long long *offs_k = nullptr;       // 3 x 3 x nomega: GEMM offsets of R1^H, R2^H, Rpg^H per point
    // spatial-ERI exchange form
    double *EK = nullptr;              // EK[(i n + k) n^2 + l n + j] = (il|kj), FP64 back-end
    double *Gp = nullptr;              // streamed form: Gram block of one panel, G[(i - i0) n + l][k n + j]
    double *EKp = nullptr;             // streamed FP64 form: the panel's exchange rows (ipanel n x n^2)
    signed char *EKpsl = nullptr;      // streamed tensor-core form: the panel's exchange rows, sliced
    int *eEKp = nullptr;
    signed char *EKsl = nullptr;       // its int8 slices, Ozaki back-end
    int *ea = nullptr, *eb = nullptr, *ozerr = nullptr;
    zc *Rho = nullptr, *Pvec = nullptr, *dvec = nullptr, *Jvec = nullptr, *Kin = nullptr, *Kvec = nullptr, *Gam = nullptr;
    signed char *Bsl = nullptr;
    // Coulomb term on the tensor cores: d = B vec P, J = B^T d (B = Cholesky vectors as L x n^2)
    signed char *B1sl = nullptr, *B2sl = nullptr, *Psl = nullptr, *dsl = nullptr;
    int *eB1 = nullptr, *eB2 = nullptr, *ePc = nullptr, *edc = nullptr;
    // int8 density GEMM (n > 64): rows (i, w) of X as an (M b) x 2N real matrix and the bra's
    // 2M x 2N real operand, sliced; rho_i8 when the plan forms rho this way
    bool rho_i8 = false;
    signed char *Xsl = nullptr, *BRsl = nullptr;
    // F X on the int8 path (fx_i8): points in sub-batches of fx_b, slices of X's columns and F's rows
    bool fx_i8 = false;
    int fx_b = 0;
    long long fx_a_rows = 0, fx_b_rows = 0;
    signed char *XTsl = nullptr, *FXsl = nullptr;
    int *eXT = nullptr, *eFX = nullptr;
    int *eX = nullptr, *eBR = nullptr;
    double *BRop = nullptr;
    double *dT = nullptr, *Jr = nullptr, *dpart = nullptr;  // dpart: split-k partials of d^T
    ~PlanImpl();
};


// buildsc.cu: BuildSC (PHF_fort/PHFTools.f90:464-537) with host arrays in the reference's layouts
// pcc.cu: PbarHbarOlap (SUCCSD_Boson_cmplx/FPUCC.f90:14-272) with host arrays in the reference's layouts
struct PccArgs {
    const phf_complex *hone, *htwo, *t1, *t2;
    int nocc, nso;
    double enuc;
    int qj, sp;
    const int *npoints;
    int npg, ncisp, ncipg, ncik;
    const phf_complex *r1, *r2, *rpg, *rk;
    const double *roota, *rootb, *rooty, *weightsp, *weightpg;
    const phf_complex *fsp, *fpg, *fk;
    int trunode;
    size_t workspace;
};
int pbarhbarolap_run(const PccArgs &g, phf_complex *olap0, phf_complex *olapex1, phf_complex *olapex2,
                     phf_complex *eolap0, phf_complex *eolapex1, phf_complex *eolapex2);

int buildsc_run(phf_complex c0, const phf_complex *c1, const phf_complex *c2, int nocc, int nso, const int *ngrid,
                int npg, const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const double *weightsp,
                const double *weightpg, int ncisp, int ncipg, const phf_complex *fsp, const phf_complex *fpg,
                size_t workspace, phf_complex *t0, phf_complex *t1, phf_complex *t2);

// phf_engine.cu
int plan_eval_batch(PlanImpl *const *plans, int count, const zc *const *d_c, zc *const *d_hs, zc *const *d_yg,
                    zc *const *d_yr, cudaStream_t st);
void plan_destroyed();  // invalidates cached batch graphs
int batch_branches();   // concurrent branches of the last captured batch graph
int profile_enable(int on);
int profile_read(int cls, double *ms, unsigned long long *count);
int plan_create(const phf_plan_desc *d, phf_plan **out);
void plan_release(PlanImpl &p);
int plan_buildhsg(PlanImpl &p, const phf_complex *z, phf_complex *hmat, phf_complex *smat, phf_complex *gradmat,
                  phf_complex *rdmmat);
int plan_eval_device(PlanImpl &p, const zc *d_c, zc *d_hs, zc *d_yg, zc *d_yr, cudaStream_t st);
int plan_eval_device_async(PlanImpl &p, const zc *d_c, zc *d_hs, zc *d_yg, zc *d_yr, int *d_status,
                           cudaStream_t st);

}  // namespace phf

struct phf_plan {
    phf::PlanImpl impl;
};
