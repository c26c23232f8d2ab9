// mixed.cu -- the mixed-precision path (FP32 fields and weights, hi/lo weights at order >= 8).
#include "internal.cuh"

namespace sunset {

int make_mixed_weights(Handle *H) {
    return set_err(H, SUNSET_ERR_SCOPE, "mixed precision is not available in this build");
}

}  // namespace sunset
