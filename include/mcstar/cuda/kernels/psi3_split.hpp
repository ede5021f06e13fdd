// call_kernel_psi3_split of mcstar-libs cuda/kernels/psi3_split.hpp:15-26: in place,
// psi -> (psi/s)^3 - psi/s - mu (+ pot), s = number of cells when norm is set else 1.
// Forwarded to pfc_psi3_split; uses the caller's Float and GPUArray typedefs.
#pragma once
#include "../../pfc_shim.hpp"

inline void call_kernel_psi3_split(GPUArray& arr, GPUArray* pot = nullptr, Float mu = Float(0), bool norm = false) {
    pfc_ctx* c = pfc_shim::context<Float>(arr.real_vext());
    PFC_SHIM_CHECK(pfc_psi3_split(c, arr.ptr_void(), pot ? pot->ptr_void() : nullptr, (double)mu, norm ? 1 : 0), c);
    PFC_SHIM_SYNC();
}
