// extern "C" entry points (include/phf_b200.h) and the LocalG kernel.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <complex>
#include <memory>
#include <string>
#include <vector>

#include "phf_internal.h"

namespace phf {

std::string &last_error_string();

namespace {

constexpr int NT = 256;

// G[ij] = (sum_t cg_t op_t(Grad[slot_t, ij]) - e0 sum_t cr_t op_t(Rdm[slot_t, ij])) / ovlp,
// op_t = identity or complex conjugate, Grad/Rdm in the (nci, nci, M, M) Fortran layout.
__global__ void localg_kernel(int MM, int nterm, const zc *cg, const zc *cr, const long long *slot, const int *cj,
                              const zc *grad, const zc *rdm, long long nslot, zc e0, zc ovlp, zc *G) {
    for (long long ij = blockIdx.x * (long long)NT + threadIdx.x; ij < MM; ij += (long long)gridDim.x * NT) {
        zc g = mkz(0, 0), r = mkz(0, 0);
        for (int t = 0; t < nterm; ++t) {
            zc a = grad[slot[t] + nslot * ij], b = rdm[slot[t] + nslot * ij];
            if (cj[t]) {
                a = conjz(a);
                b = conjz(b);
            }
            g = g + cg[t] * a;
            r = r + cr[t] * b;
        }
        G[ij] = divz(g - e0 * r, ovlp);
    }
}

}  // namespace

int launch_localg(int MM, int nterm, const zc *coef_g, const zc *coef_r, const long long *slot_of_term,
                  const int *conj_of_term, const zc *gradmat, const zc *rdmmat, long long nslot, zc e0, zc ovlp, zc *G,
                  cudaStream_t st) {
    int grid = (MM + NT - 1) / NT;
    if (grid > 148 * 8) grid = 148 * 8;
    localg_kernel<<<grid, NT, 0, st>>>(MM, nterm, coef_g, coef_r, slot_of_term, conj_of_term, gradmat, rdmmat, nslot,
                                        e0, ovlp, G);
    ++g_launches;
    PHF_CHECK_LAUNCH();
    return PHF_OK;
}

}  // namespace phf

using phf::cd;

namespace {

const char *kVersion = "phf_b200 0.1 (sm_100a)";

int fill_desc(phf_plan_desc &d, int nso, int nocc, const int *ngrid, int npg, int nci, int cmplxconj, int ncisp,
              int ncipg, const phf_complex *ref, const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg,
              const double *weightsp, const double *weightpg, const double *roota, const double *rootb,
              const double *rooty, int qj, int sp) {
    std::memset(&d, 0, sizeof(d));
    d.nso = nso;
    d.nocc = nocc;
    d.ref = ref;
    d.ngrid = ngrid;
    d.npg = npg;
    d.nci = nci;
    d.ncisp = ncisp;
    d.ncipg = ncipg;
    d.cmplxconj = cmplxconj;
    d.qj = qj;
    d.sp = sp;
    d.r1 = r1;
    d.r2 = r2;
    d.rpg = rpg;
    d.weightsp = weightsp;
    d.weightpg = weightpg;
    d.roota = roota;
    d.rootb = rootb;
    d.rooty = rooty;
    return PHF_OK;
}

}  // namespace

extern "C" {

int phf_buildhsg(const phf_complex *hone, const phf_complex *htwo, const phf_complex *ref, const phf_complex *z,
                 const int *ngrid, int npg, int nci, int cmplxconj, int ncisp, int ncipg, int nocc, int nso,
                 const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const double *weightsp,
                 const double *weightpg, const double *roota, const double *rootb, const double *rooty, int qj,
                 int sp, phf_complex *hmat, phf_complex *smat, phf_complex *gradmat, phf_complex *rdmmat) {
    phf::set_error(PHF_OK, "");
    if (!z || !hmat || !smat || !gradmat || !rdmmat) {
        phf::set_error(PHF_ERR_ARG, "null buffer");
        return PHF_ERR_ARG;
    }
    phf_plan_desc d;
    fill_desc(d, nso, nocc, ngrid, npg, nci, cmplxconj, ncisp, ncipg, ref, r1, r2, rpg, weightsp, weightpg, roota, rootb,
              rooty, qj, sp);
    d.hone = hone;
    d.htwo = htwo;
    d.precision = PHF_PREC_FP64;
    phf_plan *plan = nullptr;
    int st = phf::plan_create(&d, &plan);
    if (st != PHF_OK) return st;
    st = phf::plan_buildhsg(plan->impl, z, hmat, smat, gradmat, rdmmat);
    phf_plan_destroy(plan);
    return st;
}

int phf_buildhsg_chol(const double *h, const double *bvec, int nchol, const phf_complex *ref, const phf_complex *z,
                      const int *ngrid, int npg, int nci, int cmplxconj, int ncisp, int ncipg, int nocc, int nso,
                      const phf_complex *r1, const phf_complex *r2, const phf_complex *rpg, const double *weightsp,
                      const double *weightpg, const double *roota, const double *rootb, const double *rooty, int qj,
                      int sp, int precision, phf_complex *hmat, phf_complex *smat, phf_complex *gradmat,
                      phf_complex *rdmmat) {
    phf::set_error(PHF_OK, "");
    if (!z || !hmat || !smat || !gradmat || !rdmmat || nchol <= 0) {
        phf::set_error(PHF_ERR_ARG, "null buffer or nchol <= 0");
        return PHF_ERR_ARG;
    }
    phf_plan_desc d;
    fill_desc(d, nso, nocc, ngrid, npg, nci, cmplxconj, ncisp, ncipg, ref, r1, r2, rpg, weightsp, weightpg, roota, rootb,
              rooty, qj, sp);
    d.nchol = nchol;
    d.h = h;
    d.bvec = bvec;
    d.precision = precision;
    phf_plan *plan = nullptr;
    int st = phf::plan_create(&d, &plan);
    if (st != PHF_OK) return st;
    st = phf::plan_buildhsg(plan->impl, z, hmat, smat, gradmat, rdmmat);
    phf_plan_destroy(plan);
    return st;
}

int phf_localg(const phf_complex *gradmat, const phf_complex *rdmmat, const phf_complex *smat, phf_complex e0, int nso,
               const phf_complex *fsp, const phf_complex *fpg, const phf_complex *fk, int nci, int ncisp, int ncipg,
               int cmplxconj, phf_complex *g) {
    phf::set_error(PHF_OK, "");
    if (!gradmat || !rdmmat || !smat || !fsp || !fpg || !fk || !g || nso <= 0 || nci <= 0) {
        phf::set_error(PHF_ERR_ARG, "null buffer or bad size");
        return PHF_ERR_ARG;
    }
    const int ncik = cmplxconj == 2 ? 2 : 1;
    if (nci != ncisp * ncipg * ncik) {
        phf::set_error(PHF_ERR_ARG, "nci != ncisp * ncipg * ncik");
        return PHF_ERR_ARG;
    }
    int dev = 0;
    {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            phf::set_error(PHF_ERR_NO_DEVICE, "no CUDA device available");
            return PHF_ERR_NO_DEVICE;
        }
        cudaGetDevice(&dev);
    }
    auto C = [](const phf_complex &a) { return cd(a.re, a.im); };
    // coefficient list of PHFTools.f90:215-245
    std::vector<cd> cg, cr;
    std::vector<long long> slot;
    std::vector<int> cj;
    cd ovlp = 0;
    const int d = ncisp * ncipg;
    auto S = [&](int m, int n) { return C(smat[(size_t)m + (size_t)nci * n]); };
    for (int ni = 0; ni < ncisp; ++ni)
        for (int nj = 0; nj < ncisp; ++nj)
            for (int p = 0; p < ncipg; ++p)
                for (int q = 0; q < ncipg; ++q) {
                    int m = ni + p * ncisp, n = nj + q * ncisp;
                    cd f = std::conj(C(fsp[ni])) * C(fsp[nj]) * std::conj(C(fpg[p])) * C(fpg[q]);
                    cd f00 = f * std::conj(C(fk[0])) * C(fk[0]);
                    cg.push_back(f00);
                    cr.push_back(f00);
                    slot.push_back(m + (long long)nci * n);
                    cj.push_back(0);
                    ovlp += f00 * S(m, n);
                    if (cmplxconj == 2) {
                        cd f11 = f * std::conj(C(fk[1])) * C(fk[1]);
                        cd f01 = f * std::conj(C(fk[0])) * C(fk[1]);
                        cd f10 = f * std::conj(C(fk[1])) * C(fk[0]);
                        cg.push_back(f11); cr.push_back(f11); slot.push_back((m + d) + (long long)nci * (n + d)); cj.push_back(1);
                        cg.push_back(f01); cr.push_back(f01); slot.push_back(m + (long long)nci * (n + d)); cj.push_back(0);
                        cg.push_back(f01); cr.push_back(f01); slot.push_back((m + d) + (long long)nci * n); cj.push_back(1);
                        ovlp += f11 * S(m + d, n + d) + f01 * S(m, n + d) + f10 * S(m + d, n);
                    }
                }
    const long long MM = (long long)nso * nso, ns = (long long)nci * nci;
    const int nterm = (int)cg.size();
    phf::zc *dg = nullptr, *dr = nullptr, *dG = nullptr, *dcg = nullptr, *dcr = nullptr;
    long long *dslot = nullptr;
    int *dcj = nullptr;
    int st = PHF_OK;
    auto fail = [&](const char *what, cudaError_t e) {
        phf::set_error(PHF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        st = PHF_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&dg, ns * MM * sizeof(phf::zc))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dr, ns * MM * sizeof(phf::zc))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dG, MM * sizeof(phf::zc))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dcg, nterm * sizeof(phf::zc))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dcr, nterm * sizeof(phf::zc))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dslot, nterm * sizeof(long long))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st && (e = cudaMalloc(&dcj, nterm * sizeof(int))) != cudaSuccess) fail("cudaMalloc", e);
    if (!st) {
        cudaMemcpy(dg, gradmat, ns * MM * sizeof(phf::zc), cudaMemcpyHostToDevice);
        cudaMemcpy(dr, rdmmat, ns * MM * sizeof(phf::zc), cudaMemcpyHostToDevice);
        cudaMemcpy(dcg, cg.data(), nterm * sizeof(phf::zc), cudaMemcpyHostToDevice);
        cudaMemcpy(dcr, cr.data(), nterm * sizeof(phf::zc), cudaMemcpyHostToDevice);
        cudaMemcpy(dslot, slot.data(), nterm * sizeof(long long), cudaMemcpyHostToDevice);
        cudaMemcpy(dcj, cj.data(), nterm * sizeof(int), cudaMemcpyHostToDevice);
        st = phf::launch_localg((int)MM, nterm, dcg, dcr, dslot, dcj, dg, dr, ns, phf::zc{e0.re, e0.im},
                                phf::zc{ovlp.real(), ovlp.imag()}, dG, 0);
        if (!st && (e = cudaMemcpy(g, dG, MM * sizeof(phf::zc), cudaMemcpyDeviceToHost)) != cudaSuccess)
            fail("cudaMemcpy", e);
    }
    cudaFree(dg);
    cudaFree(dr);
    cudaFree(dG);
    cudaFree(dcg);
    cudaFree(dcr);
    cudaFree(dslot);
    cudaFree(dcj);
    return st;
}

int phf_plan_create(const phf_plan_desc *desc, phf_plan **plan) {
    phf::set_error(PHF_OK, "");
    if (!plan) {
        phf::set_error(PHF_ERR_ARG, "null plan pointer");
        return PHF_ERR_ARG;
    }
    return phf::plan_create(desc, plan);
}

int phf_plan_destroy(phf_plan *plan) {
    if (plan) phf::plan_destroyed();  // batch graphs that contain it are recaptured
    delete plan;                      // ~PlanImpl releases the device memory and library handles
    return PHF_OK;
}

int phf_batch_branches(void) { return phf::batch_branches(); }

int phf_eval_batch(phf_plan *const *plans, int count, const phf_complex *const *d_c, phf_complex *const *d_hs,
                   phf_complex *const *d_yg, phf_complex *const *d_yr, void *stream) {
    phf::set_error(PHF_OK, "");
    if (count < 0 || (count > 0 && (!plans || !d_c || !d_hs || !d_yg || !d_yr))) {
        phf::set_error(PHF_ERR_ARG, "phf_eval_batch: null argument");
        return PHF_ERR_ARG;
    }
    std::vector<phf::PlanImpl *> impl((size_t)count);
    for (int i = 0; i < count; ++i) {
        if (!plans[i] || !d_c[i] || !d_hs[i] || !d_yg[i] || !d_yr[i]) {
            phf::set_error(PHF_ERR_ARG, "phf_eval_batch: null plan or buffer at index " + std::to_string(i));
            return PHF_ERR_ARG;
        }
        impl[i] = &plans[i]->impl;
    }
    return phf::plan_eval_batch(impl.data(), count, reinterpret_cast<const phf::zc *const *>(d_c),
                                reinterpret_cast<phf::zc *const *>(d_hs), reinterpret_cast<phf::zc *const *>(d_yg),
                                reinterpret_cast<phf::zc *const *>(d_yr), reinterpret_cast<cudaStream_t>(stream));
}

int phf_plan_buildhsg(phf_plan *plan, const phf_complex *z, phf_complex *hmat, phf_complex *smat,
                      phf_complex *gradmat, phf_complex *rdmmat) {
    phf::set_error(PHF_OK, "");
    if (!plan || !z || !hmat || !smat || !gradmat || !rdmmat) {
        phf::set_error(PHF_ERR_ARG, "null argument");
        return PHF_ERR_ARG;
    }
    return phf::plan_buildhsg(plan->impl, z, hmat, smat, gradmat, rdmmat);
}

int phf_plan_eval_device(phf_plan *plan, const phf_complex *d_c, phf_complex *d_hs, phf_complex *d_yg,
                         phf_complex *d_yr, void *stream) {
    phf::set_error(PHF_OK, "");
    if (!plan || !d_c || !d_hs || !d_yg || !d_yr) {
        phf::set_error(PHF_ERR_ARG, "null argument");
        return PHF_ERR_ARG;
    }
    return phf::plan_eval_device(plan->impl, reinterpret_cast<const phf::zc *>(d_c), reinterpret_cast<phf::zc *>(d_hs),
                                 reinterpret_cast<phf::zc *>(d_yg), reinterpret_cast<phf::zc *>(d_yr),
                                 reinterpret_cast<cudaStream_t>(stream));
}

int phf_plan_eval_device_async(phf_plan *plan, const phf_complex *d_c, phf_complex *d_hs, phf_complex *d_yg,
                               phf_complex *d_yr, int *d_status, void *stream) {
    phf::set_error(PHF_OK, "");
    if (!plan || !d_c || !d_hs || !d_yg || !d_yr || !d_status) {
        phf::set_error(PHF_ERR_ARG, "null argument");
        return PHF_ERR_ARG;
    }
    return phf::plan_eval_device_async(plan->impl, reinterpret_cast<const phf::zc *>(d_c),
                                       reinterpret_cast<phf::zc *>(d_hs), reinterpret_cast<phf::zc *>(d_yg),
                                       reinterpret_cast<phf::zc *>(d_yr), d_status,
                                       reinterpret_cast<cudaStream_t>(stream));
}

int phf_tuned_shapes(void) { return phf::tuned_entries(); }

int phf_int8_wide_mma(int on) {
    const int was = !phf::g_narrow_mma;
    phf::g_narrow_mma = on ? 0 : 1;
    return was;
}

int phf_int8_fock_product(int on) {
    const int was = phf::g_fx_i8;
    phf::g_fx_i8 = on > 0 ? on : 0;
    return was;
}

int phf_buildsc(phf_complex c0, const phf_complex *c1, const phf_complex *c2, int nocc, int nso, const int *ngrid,
                int npg, int qj, int ncisp, int ncipg, int ncik, const phf_complex *r1, const phf_complex *r2,
                const phf_complex *rpg, const phf_complex *rk, const double *roota, const double *rootb,
                const double *rooty, const double *weightsp, const double *weightpg, const phf_complex *fsp,
                const phf_complex *fpg, const phf_complex *fk, phf_complex *t0, phf_complex *t1, phf_complex *t2) {
    (void)qj, (void)ncik, (void)rk, (void)roota, (void)rootb, (void)rooty, (void)fk;
    phf::set_error(PHF_OK, "");
    if (!c1 || !c2 || !ngrid || !r1 || !r2 || !rpg || !weightsp || !weightpg || !fsp || !fpg || !t0 || !t1 || !t2 ||
        nso <= 0 || nocc <= 0 || nocc > nso || ngrid[0] <= 0 || ngrid[1] <= 0 || npg <= 0 || ncisp <= 0 ||
        ncipg <= 0) {
        phf::set_error(PHF_ERR_ARG, "phf_buildsc: missing or non-positive argument");
        return PHF_ERR_ARG;
    }
    if (nocc > phf::kMaxOverlapN) {
        phf::set_error(PHF_ERR_UNSUPPORTED, "phf_buildsc: nocc above the overlap inverse's limit");
        return PHF_ERR_UNSUPPORTED;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        phf::set_error(PHF_ERR_NO_DEVICE, "no CUDA device available");
        return PHF_ERR_NO_DEVICE;
    }
    return phf::buildsc_run(c0, c1, c2, nocc, nso, ngrid, npg, r1, r2, rpg, weightsp, weightpg, ncisp, ncipg, fsp,
                            fpg, 0, t0, t1, t2);
}

int phf_plan_info(const phf_plan *plan, int *chunk, size_t *workspace_bytes) {
    if (!plan) return PHF_ERR_ARG;
    if (chunk) *chunk = plan->impl.b;
    if (workspace_bytes) *workspace_bytes = plan->impl.arena.total;
    return PHF_OK;
}

const char *phf_status_string(int status) {
    switch (status) {
        case PHF_OK: return "ok";
        case PHF_ERR_ARG: return "invalid argument";
        case PHF_ERR_SINGULAR: return "singular rotated overlap";
        case PHF_ERR_NOT_HERMITIAN: return "Hmat/Smat not Hermitian";
        case PHF_ERR_NONFINITE: return "non-finite value";
        case PHF_ERR_CUDA: return "CUDA error";
        case PHF_ERR_OOM: return "device out of memory";
        case PHF_ERR_UNSUPPORTED: return "unsupported option or size";
        case PHF_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char *phf_last_error(void) { return phf::last_error_string().c_str(); }

unsigned long long phf_kernel_launches(void) { return phf::g_launches; }

int phf_profile_enable(int on) { return phf::profile_enable(on); }

int phf_profile_read(int kernel_class, double *total_ms, unsigned long long *launches) {
    if (kernel_class < 0 || kernel_class >= phf::PROF_NCLASS) return PHF_ERR_ARG;
    return phf::profile_read(kernel_class, total_ms, launches);
}

const char *phf_version(void) { return kVersion; }

}  // extern "C"
