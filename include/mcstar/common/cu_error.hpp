// CUERR as in mcstar-libs common/cu_error.hpp:3-11: a failed CUDA runtime call prints
// its error string with the call site and ends the process with the error code.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

namespace CUERROR {
inline void gpuAssert(cudaError_t code, const char* file, int line) {
    if (code != cudaSuccess) {
        fprintf(stderr, "CUERR: %s %s:%d\n", cudaGetErrorString(code), file, line);
        fflush(stderr);
        exit(code);
    }
}
}  // namespace CUERROR

#define CUERR(ans) CUERROR::gpuAssert((ans), __FILE__, __LINE__);
