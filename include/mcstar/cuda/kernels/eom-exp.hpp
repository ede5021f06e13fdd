// The exponential (integrating-factor) conserved update of mcstar-libs
// cuda/kernels/eom-exp.hpp:3-90: call_kernel_init_eom_op, the kop overloads of
// call_kernel_update_eom / call_kernel_update_eom_with_fen, and call_kernel_calc_fen
// (here over the whole real field; the reference launches it over the complex extent).
// Forwarded to pfc_init_eom_op / pfc_update_eom_exp(_with_fen) / pfc_calc_fen.  Uses
// the caller's Float, Float3 and GPUArray typedefs; like the reference it cannot share a
// translation unit with eom.hpp (both define call_kernel_calc_fen).
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_init_eom_op(GPUArray& arr_kop, Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kop.real_vext());
    PFC_SHIM_CHECK(pfc_init_eom_op(c, arr_kop.ptr_void(), dt, eps, lens.x, lens.y, lens.z), c);
    PFC_SHIM_SYNC();
}

inline void call_kernel_update_eom(GPUArray& arr_kop, GPUArray& arr_kpsi, GPUArray& arr_knonlin, GPUArray& arr_knoise,
                                   Float namp, Float dt, Float eps, Float3 lens) {
    (void)dt;
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_exp(c, arr_kop.ptr_void(), arr_kpsi.ptr_void(), arr_knonlin.ptr_void(),
                                      arr_knoise.ptr_void(), namp, eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

inline void call_kernel_update_eom(GPUArray& arr_kop, GPUArray& arr_kpsi, GPUArray& arr_knonlin, Float namp, Float dt,
                                   Float eps, Float3 lens) {
    (void)dt;
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_exp(c, arr_kop.ptr_void(), arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), nullptr,
                                      namp, eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

inline void call_kernel_update_eom_with_fen(GPUArray& arr_kop, GPUArray& arr_kpsi, GPUArray& arr_knonlin,
                                            GPUArray& arr_knoise, Float namp, Float dt, Float eps, Float3 lens) {
    (void)dt;
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_exp_with_fen(c, arr_kop.ptr_void(), arr_kpsi.ptr_void(), arr_knonlin.ptr_void(),
                                               arr_knoise.ptr_void(), namp, eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

inline float call_kernel_calc_fen(GPUArray& arr_psi, GPUArray& arr_lpsi, Float3 hh) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_psi.real_vext());
    double f = 0.0;
    PFC_SHIM_CHECK(pfc_calc_fen(c, arr_psi.ptr_void(), arr_lpsi.ptr_void(), hh.x, hh.y, hh.z, &f), c);
    PFC_SHIM_SYNC();
    return (float)f;
}
