// The exponential form of the non-conserved relaxation, mcstar-libs
// cuda/kernels/el-exp.hpp:3-60: call_kernel_init_el_op builds kop = {exp(-L dt),
// (exp(-L dt) - 1)/L}, L = (1 - k^2)^2 + 1 - eps; call_kernel_update_el(kop, ...) applies
// psi^ <- kop.x psi^ + kop.y N^ and returns the largest mode change.  Forwarded to
// pfc_init_el_op / pfc_update_el_exp; uses the caller's typedefs.
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_init_el_op(GPUArray& arr_kop, Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kop.real_vext());
    PFC_SHIM_CHECK(pfc_init_el_op(c, arr_kop.ptr_void(), dt, eps, lens.x, lens.y, lens.z), c);
    PFC_SHIM_SYNC();
}

inline Float call_kernel_update_el(GPUArray& arr_kop, GPUArray& arr_kpsi, GPUArray& arr_knonlin, Float dt, Float eps,
                                   Float3 lens) {
    (void)dt;
    (void)eps;
    (void)lens;
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    double m = 0.0;
    PFC_SHIM_CHECK(pfc_update_el_exp(c, arr_kop.ptr_void(), arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), &m), c);
    PFC_SHIM_SYNC();
    return (Float)m;
}
