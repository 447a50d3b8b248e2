// Tensor-core (mixed-precision) form of the kinship operator.
#include "cs_internal.h"

namespace cs {

struct MixedOperator {};

void destroy_mixed(MixedOperator* m) { delete m; }

void kinship_apply_mixed(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                         int64_t ldy, cudaStream_t s) {
    (void)op; (void)X; (void)ldx; (void)k; (void)Y; (void)ldy; (void)s;
    fail(CS_ERR_UNSUPPORTED, "mixed-precision operator not built yet");
}

}  // namespace cs
