// FFT::CufftPlan<F, R2C|C2R> with the interface of mcstar-libs
// cuda/cufft_wrapper.hpp:40-86, executed by libpfc_b200's own register-resident
// transforms (pfc_fft_r2c / pfc_fft_c2r) instead of cuFFT.  Unnormalised like
// cuFFT: a round trip multiplies by the number of cells.  The input array is left
// unchanged by both directions.
#pragma once
#include <cassert>

#include "../pfc_shim.hpp"
#include "array_abstraction.hpp"

namespace FFT {

struct R2C {};
struct C2R {};

template <typename F, typename FT> class CufftPlan {
    int3 m_shape;
    pfc_ctx* m_ctx;

    void run(Array::GPUArray<F>& in, Array::GPUArray<F>& out, R2C) {
        PFC_SHIM_CHECK(pfc_fft_r2c(m_ctx, in.ptr_void(), out.ptr_void()), m_ctx);
    }
    void run(Array::GPUArray<F>& in, Array::GPUArray<F>& out, C2R) {
        PFC_SHIM_CHECK(pfc_fft_c2r(m_ctx, in.ptr_void(), out.ptr_void()), m_ctx);
    }

  public:
    // the logical (real) extent, x fastest
    explicit CufftPlan(int3 shape) : m_shape(shape), m_ctx(pfc_shim::context<F>(shape)) {}
    void execute(Array::GPUArray<F>& in, Array::GPUArray<F>& out) {
        assert(in.real_vext() == m_shape && out.real_vext() == m_shape &&
               "array dimensions in plan and execute phase do not match up");
        assert(in.ptr_void() != out.ptr_void() && "in-place transforms are not supported");
        run(in, out, FT{});
        PFC_SHIM_SYNC();
    }
};

}  // namespace FFT
