// The non-conserved semi-implicit relaxation of mcstar-libs cuda/kernels/el.hpp:3-45:
// psi^ <- (psi^ - dt N^)/(1 + dt((1 - k^2)^2 + 1 - eps)); returns max_k |psi^'_k - psi^_k|
// (used by the reference's drivers as the convergence measure).  Forwarded to
// pfc_update_el; uses the caller's Float, Float3 and GPUArray typedefs.
#pragma once
#include "../../pfc_shim.hpp"

inline Float call_kernel_update_el(GPUArray& arr_kpsi, GPUArray& arr_knonlin, Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    double m = 0.0;
    PFC_SHIM_CHECK(pfc_update_el(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), dt, eps, lens.x, lens.y, lens.z, &m),
                   c);
    PFC_SHIM_SYNC();
    return (Float)m;
}
