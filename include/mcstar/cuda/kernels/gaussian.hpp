// The Gaussian filter of mcstar-libs cuda/kernels/gaussian.hpp:23-67:
// call_kernel_gaussian_init writes kgauss_k = (e, 1 - e), e = exp(-1/2 sum_a (1.1 d h_a K_a)^2)
// (the low-pass in the real part, the complementary high-pass in the imaginary part);
// call_kernel_kmult_real / _imag multiply a half spectrum by one of them.  Forwarded to
// pfc_gaussian_init / pfc_kmult_real / pfc_kmult_imag; uses the caller's Float, Float3 and
// GPUArray typedefs.
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_gaussian_init(GPUArray& arr_kpsi, Float3 lens, Float3 hh, Float divs_per_sigma) {
    pfc_ctx* c = pfc_shim::context<Float>(arr_kpsi.real_vext());
    PFC_SHIM_CHECK(pfc_gaussian_init(c, arr_kpsi.ptr_void(), lens.x, lens.y, lens.z, hh.x, hh.y, hh.z, divs_per_sigma),
                   c);
    PFC_SHIM_SYNC();
}

inline void call_kernel_kmult_real(GPUArray& arr_1, GPUArray& arr_2) {
    assert(arr_1.real_vext() == arr_2.real_vext() && "array dimensions do not match");
    pfc_ctx* c = pfc_shim::context<Float>(arr_1.real_vext());
    PFC_SHIM_CHECK(pfc_kmult_real(c, arr_1.ptr_void(), arr_2.ptr_void()), c);
    PFC_SHIM_SYNC();
}

inline void call_kernel_kmult_imag(GPUArray& arr_1, GPUArray& arr_2) {
    assert(arr_1.real_vext() == arr_2.real_vext() && "array dimensions do not match");
    pfc_ctx* c = pfc_shim::context<Float>(arr_1.real_vext());
    PFC_SHIM_CHECK(pfc_kmult_imag(c, arr_1.ptr_void(), arr_2.ptr_void()), c);
    PFC_SHIM_SYNC();
}
