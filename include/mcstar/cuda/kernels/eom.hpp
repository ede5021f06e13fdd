// The conserved semi-implicit update and the free-energy density of mcstar-libs
// cuda/kernels/eom.hpp:60-141 (call_kernel_update_eom, call_kernel_update_eom_with_fen,
// call_kernel_calc_fen), forwarded to pfc_update_eom / pfc_update_eom_with_fen /
// pfc_calc_fen.  Uses the caller's typedefs Float, Float3 and GPUArray (as the
// reference does), so include it after them.  calc_fen sums in FP64 in a fixed
// order, so repeated calls agree exactly (the reference sums float atomics).
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_update_eom(GPUArray& arr_kpsi, GPUArray& arr_knonlin, GPUArray& arr_knoise, Float namp,
                                   Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), arr_knoise.ptr_void(), namp, dt,
                                  eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

// without noise (eom.hpp:80-86)
inline void call_kernel_update_eom(GPUArray& arr_kpsi, GPUArray& arr_knonlin, Float namp, Float dt, Float eps,
                                   Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), nullptr, namp, dt, eps, lens.x,
                                  lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

// also overwrites arr_knoise with L^ psi^ of the state before the update
inline void call_kernel_update_eom_with_fen(GPUArray& arr_kpsi, GPUArray& arr_knonlin, GPUArray& arr_knoise,
                                            Float namp, Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_with_fen(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), arr_knoise.ptr_void(),
                                           namp, dt, eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

// the update with the polynomial kernel P(k^2) (eom.hpp:143-180)
inline void call_kernel_update_eom_py(GPUArray& arr_kpsi, GPUArray& arr_knonlin, GPUArray& arr_knoise, Float namp,
                                      Float dt, Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_py(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), arr_knoise.ptr_void(), namp, dt,
                                     eps, lens.x, lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

// the 2D update with anisotropic noise from three noise fields (eom.hpp:16-58)
inline void call_kernel_update_eom_hpfcnoise(GPUArray& arr_kpsi, GPUArray& arr_knonlin, GPUArray& arr_knoise1,
                                             GPUArray& arr_knoise2, GPUArray& arr_knoise3, Float namp, Float dt,
                                             Float eps, Float3 lens) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_update_eom_hpfcnoise(c, arr_kpsi.ptr_void(), arr_knonlin.ptr_void(), arr_knoise1.ptr_void(),
                                            arr_knoise2.ptr_void(), arr_knoise3.ptr_void(), namp, dt, eps, lens.x,
                                            lens.y, lens.z),
                   c);
    PFC_SHIM_SYNC();
}

// writes f = psi (L psi - psi + psi^3 / 2) / 2 into arr_lpsi; returns h^3 sum(f)
inline float call_kernel_calc_fen(GPUArray& arr_psi, GPUArray& arr_lpsi, Float3 hh) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_psi.real_vext());
    double f = 0.0;
    PFC_SHIM_CHECK(pfc_calc_fen(c, arr_psi.ptr_void(), arr_lpsi.ptr_void(), hh.x, hh.y, hh.z, &f), c);
    PFC_SHIM_SYNC();
    return (float)f;
}
