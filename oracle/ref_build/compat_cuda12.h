/* Compatibility shim force-included when compiling the reference's CUDA headers
 * with CUDA 12.9.  The reference was written for CUDA <= 8:
 *   - cufftSetCompatibilityMode / CUFFT_COMPATIBILITY_NATIVE were removed from
 *     cuFFT (reference cuda/cufft_wrapper.hpp:77); native layout is now the only
 *     layout, so the call becomes a no-op that reports success;
 *   - cudaThreadSynchronize was removed (used after every reference launch);
 *     cudaDeviceSynchronize is its documented replacement.
 * Nothing else of the reference is changed.  Test infrastructure only. */
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <cassert>
#include <cstring>
#define CUFFT_COMPATIBILITY_NATIVE 0
#define cufftSetCompatibilityMode(plan, mode) CUFFT_SUCCESS
#define cudaThreadSynchronize cudaDeviceSynchronize
