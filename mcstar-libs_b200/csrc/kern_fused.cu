// Fused plane kernels of the stepper (filled in below the general path).
#include "pfc_ctx.h"

namespace pfc {

int fused_xy_variant(int, int, int) { return 0; }
cudaError_t set_fused_attributes(const pfc_ctx*) { return cudaSuccess; }
cudaError_t launch_fused_xy(const pfc_ctx*, const void*, void*, const void*, double, double, double) {
    return cudaErrorNotSupported;
}

}  // namespace pfc
