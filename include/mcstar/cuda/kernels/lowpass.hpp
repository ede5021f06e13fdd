// The 2D spectral low-pass post-processing of mcstar-libs cuda/kernels/lowpass.hpp:1-93:
// the multiply helpers, _call_kernel_square, write_lowpass_2d (the spectrum low-passed in
// place, then the gzip-compressed LOWPASS text dump in the reference's byte format) and
// calc_amplitude_lowpass (high-pass, square, low-pass and the dump; the amplitude field ends
// in aux and in host's real view).  Forwarded to pfc_kmult_*, pfc_square,
// pfc_write_lowpass_2d and pfc_amplitude_lowpass; uses the caller's Float, Float3,
// GPUArray, CPUArray, PlanR2C and PlanC2R typedefs.  Non-2D arrays end the program with a
// message, as the reference's asserts do.
#pragma once
#include <string>
#include "../../pfc_shim.hpp"

inline void _call_kernel_multassign_cmpl_with_real(GPUArray& karr1, GPUArray& karr2) {
    pfc_ctx* c = pfc_shim::context<Float>(karr1.real_vext());
    PFC_SHIM_CHECK(pfc_kmult_real(c, karr1.ptr_void(), karr2.ptr_void()), c);
    PFC_SHIM_SYNC();
}

inline void _call_kernel_multassign_cmpl_with_imag(GPUArray& karr1, GPUArray& karr2) {
    pfc_ctx* c = pfc_shim::context<Float>(karr1.real_vext());
    PFC_SHIM_CHECK(pfc_kmult_imag(c, karr1.ptr_void(), karr2.ptr_void()), c);
    PFC_SHIM_SYNC();
}

inline void _call_kernel_square(GPUArray& karr1) {
    pfc_ctx* c = pfc_shim::context<Float>(karr1.real_vext());
    PFC_SHIM_CHECK(pfc_square(c, karr1.ptr_void()), c);
    PFC_SHIM_SYNC();
}

inline void write_lowpass_2d(GPUArray& spectrum, GPUArray& kgaussian, CPUArray& host, Float3 ll, std::string fn) {
    (void)host;  // the library stages the copy itself
    pfc_ctx* c = pfc_shim::context<Float>(spectrum.real_vext());
    PFC_SHIM_CHECK(pfc_write_lowpass_2d(c, spectrum.ptr_void(), kgaussian.ptr_void(), ll.x, ll.y, fn.c_str()), c);
    PFC_SHIM_SYNC();
}

inline void calc_amplitude_lowpass(PlanR2C& r2c, PlanC2R& c2r, GPUArray& spectrum, GPUArray& aux,
                                   GPUArray& kgaussian, CPUArray& host, Float3 ll, std::string fn) {
    (void)r2c;
    (void)c2r;
    pfc_ctx* c = pfc_shim::context<Float>(spectrum.real_vext());
    PFC_SHIM_CHECK(pfc_amplitude_lowpass(c, spectrum.ptr_void(), aux.ptr_void(), kgaussian.ptr_void(), ll.x, ll.y,
                                         fn.c_str()),
                   c);
    PFC_SHIM_SYNC();
    aux >> host;
}
