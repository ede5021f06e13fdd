// NoiseHostApi<F> with the interface of mcstar-libs cuda/noise.hpp:93-150, drawing
// from libpfc_b200's counter-based Philox4x32-10 generator instead of cuRAND XORWOW:
// the draws have the same distributions (fill: real N(0, sigma^2) per element;
// fill_kspace: the Hermitian complex normal spectrum of noise.hpp:110-142) but not the
// same values.  Draw i of a generator made with `seed` uses counter i, so a run can be
// reproduced or resumed from (seed, number of draws).
#pragma once
#include "../pfc_shim.hpp"
#include "array_abstraction.hpp"

template <typename F> class NoiseHostApi {
    unsigned long long m_seed;
    unsigned long long m_draws;

  public:
    explicit NoiseHostApi(unsigned long long int seed = 1234L) : m_seed(seed), m_draws(0) {}
    void fill(Array::GPUArray<F>& arr, F sigma) {
        pfc_ctx* c = pfc_shim::context<F>(arr.real_vext());
        PFC_SHIM_CHECK(pfc_noise_fill(c, arr.ptr_void(), (double)sigma, m_seed, m_draws++), c);
        PFC_SHIM_SYNC();
    }
    void fill_kspace(Array::GPUArray<F>& arr) {
        pfc_ctx* c = pfc_shim::context<F>(arr.real_vext());
        PFC_SHIM_CHECK(pfc_noise_fill_kspace(c, arr.ptr_void(), m_seed, m_draws++), c);
        PFC_SHIM_SYNC();
    }
    unsigned long long draws() const { return m_draws; }
};
