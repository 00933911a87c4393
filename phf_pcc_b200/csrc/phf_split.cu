// Tensor-core hooks of the factorized (Cholesky) J/K form.  The tensor-core arithmetic of
// this version runs in the spatial-ERI exchange form (ozaki_i8.cu); the factorized form is
// FP64 only and these hooks only validate the plan.
#include "phf_internal.h"

namespace phf {

size_t split_bytes_per_point(const PlanImpl &p) {
    (void)p;
    return 0;
}

int split_setup(PlanImpl &p) {
    // the int8 tensor-core back-end of the spatial-ERI exchange form is set up with the
    // exchange matrix; the factorized form has no tensor-core back-end in this version
    if (p.prec != PHF_PREC_FP64 && !p.eri) {
        set_error(PHF_ERR_UNSUPPORTED, "tensor-core precisions need the spatial-ERI exchange form");
        return PHF_ERR_UNSUPPORTED;
    }
    return PHF_OK;
}

int split_gamma_x(PlanImpl &p, int bc, cudaStream_t st) {
    (void)p;
    (void)bc;
    (void)st;
    set_error(PHF_ERR_UNSUPPORTED, "tensor-core precisions are not built into this library version");
    return PHF_ERR_UNSUPPORTED;
}

}  // namespace phf
