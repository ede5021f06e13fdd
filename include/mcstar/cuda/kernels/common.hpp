// Index and launch helpers of mcstar-libs cuda/kernels/common.hpp:1-58, for the
// caller's own kernels: x-fastest linear index, periodic wrap, the wavenumber
// K(i) = i' 2 pi / L with i' = i for i < n/2 + 1 else i - n, the operator pair
// L_L2 = (-k^2, k^4), ceil division and the default block shapes of `Launch`.
// K and L_L2 need the caller's FLOAT / Float / Float2 definitions, as in the reference.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

// thread -> (i0, i1, i2) and its linear index idx; threads outside `dims` return
#define IDX012(dims)                                 \
    int i0 = blockIdx.x * blockDim.x + threadIdx.x;  \
    int i1 = blockIdx.y * blockDim.y + threadIdx.y;  \
    int i2 = blockIdx.z * blockDim.z + threadIdx.z;  \
    int idx = calc_idx(i0, i1, i2, dims);            \
    if (i0 >= dims.x or i1 >= dims.y or i2 >= dims.z) return;

__host__ __device__ inline int wrap(int i, int n) { return i < 0 ? (i + n) : (i >= n ? (i - n) : i); }

__forceinline__ __host__ __device__ int calc_idx(int i0, int i1, int i2, int3 dims) {
    return (i2 * dims.y + i1) * dims.x + i0;
}

#ifdef FLOAT
__forceinline__ __device__ Float2 L_L2(Float k0, Float k1, Float k2) {
    Float2 r;
    r.x = -k0 * k0 - k1 * k1 - k2 * k2;
    r.y = r.x * r.x;
    return r;
}
__forceinline__ __device__ Float K(int i, int n, Float len) {
    return (i < n / 2 + 1 ? i : i - n) * Float(6.283185307179586232) / len;
}
#endif

inline unsigned int div_up(int a, int b) { return (unsigned int)(a / b + (a % b > 0 ? 1 : 0)); }

// n mod m in [0, m) for either sign of n
__host__ __device__ inline unsigned int posrem(int n, int m) { return n - (n / m - int(n < 0)) * m; }

struct Launch {
    const dim3 bs1d = {512};
    const dim3 bs2d = {16, 32};
    const dim3 bs3d = {8, 8, 8};
    dim3 bs, gs;
    explicit Launch(int n0) : Launch(int3{n0, 1, 1}) {}
    explicit Launch(int3 shape) {
        if (shape.y == 1 && shape.z == 1) {
            bs = bs1d;
            gs = dim3(div_up(shape.x, bs.x));
        } else if (shape.z == 1) {
            bs = bs2d;
            gs = dim3(div_up(shape.x, bs.x), div_up(shape.y, bs.y));
        } else {
            bs = bs3d;
            gs = dim3(div_up(shape.x, bs.x), div_up(shape.y, bs.y), div_up(shape.z, bs.z));
        }
    }
    dim3 get_bs() { return bs; }
    dim3 get_gs() { return gs; }
};
