// Tensor-core (tcgen05) path of the Cholesky J/K contraction.  Filled in by the split-
// precision kernels; until a precision other than FP64 is requested it allocates nothing.
#include "phf_internal.h"

namespace phf {

size_t split_bytes_per_point(const PlanImpl &p) {
    (void)p;
    return 0;
}

int split_setup(PlanImpl &p) {
    if (p.prec != PHF_PREC_FP64) {
        set_error(PHF_ERR_UNSUPPORTED, "tensor-core precisions are not built into this library version");
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
