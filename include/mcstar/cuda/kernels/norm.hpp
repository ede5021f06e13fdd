// call_kernel_norm of mcstar-libs cuda/kernels/norm.hpp:5-10: divides the real field
// by its number of cells, in place.  Forwarded to pfc_norm.
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_norm(GPUArray& arr) {
    pfc_ctx* c = pfc_shim::context<Float>(arr.real_vext());
    PFC_SHIM_CHECK(pfc_norm(c, arr.ptr_void()), c);
    PFC_SHIM_SYNC();
}
