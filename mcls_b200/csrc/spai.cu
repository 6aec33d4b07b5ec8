// spai.cu -- learned sparse-approximate-inverse preconditioner.
#include "internal.h"

namespace mclsgpu {

int spai_build(mclsgpu_context* ctx, mclsgpu_operator* op, const mclsgpu_precond_params* p,
               mclsgpu_precond* pc) {
    (void)op;
    (void)p;
    (void)pc;
    return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "learned SPAI preconditioner not available");
}

}  // namespace mclsgpu
