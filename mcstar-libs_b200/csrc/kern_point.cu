// Pointwise kernels of the reference-shaped API (cuda/kernels/eom.hpp, psi3_split.hpp,
// norm.hpp, noise.hpp) and the FP64 reductions of the free energy.  All are
// grid-stride loops over the flat half spectrum or real field; they are HBM-bound.
#include "pfc_ctx.h"

namespace pfc {
namespace {

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    const size_t cap = 148 * 16;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

// |k| as the reference evaluates it, sqrtf(-dop.x) (eom.hpp:68): single precision even
// when Float is double.
template <typename T> __device__ __forceinline__ T ref_sqrtf(T x) { return (T)sqrtf((float)x); }

// kernel_update_eom / kernel_update_eom_with_fen (eom.hpp:60-72, 88-102), with the
// stabilisation constant C (C = 1 is the reference: (1 + C - eps) = (2 - eps)).
template <typename T>
__global__ void k_update_eom(cx<T>* __restrict__ kpsi, const cx<T>* __restrict__ knl, cx<T>* knoise, int nx, int ny,
                             int nz, T namp_eff, T dt, T eps, T lx, T ly, T lz, int with_fen, T C) {
    const int nxh = nx / 2 + 1;
    const int64_t total = (int64_t)nxh * ny * nz;
    const T deps = T(1) + C - eps;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % nxh);
        const int64_t r = idx / nxh;
        const int i1 = (int)(r % ny), i2 = (int)(r / ny);
        const cx<T> p = kpsi[idx];
        const cx<T> q = knl[idx];
        const cx<T> w = knoise ? knoise[idx] : mkc<T>(T(0), T(0));
        const T k0 = kwave<T>(i0, nx, lx), k1 = kwave<T>(i1, ny, ly), k2 = kwave<T>(i2, nz, lz);
        const T dopx = -k0 * k0 - k1 * k1 - k2 * k2;
        const T dopy = dopx * dopx;
        const T k = ref_sqrtf<T>(-dopx);
        T denom;
        if (with_fen) {
            const T lk = (T(2) - eps) + T(2) * dopx + dopy;
            denom = T(1) - dt * dopx * ((C - T(1)) + lk);
            knoise[idx] = mkc<T>(lk * p.x, lk * p.y);
        } else {
            denom = T(1) - dt * (deps * dopx + T(2) * dopy + dopx * dopy);
        }
        kpsi[idx] = mkc<T>((p.x + dt * dopx * q.x + dt * namp_eff * k * w.x) / denom,
                           (p.y + dt * dopx * q.y + dt * namp_eff * k * w.y) / denom);
    }
}

// kernel_psi3_split(_pot) (psi3_split.hpp:1-13) with the stabilisation constant C.
template <typename T>
__global__ void k_psi3(T* __restrict__ arr, const T* __restrict__ pot, int64_t n, T mul, T mu, T C) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T t = arr[i] * mul;
        T v = t * t * t - C * t - mu;
        if (pot) v += pot[i];
        arr[i] = v;
    }
}

// kernel_norm (norm.hpp:1-3)
template <typename T>
__global__ void k_norm(T* __restrict__ arr, int64_t n, T nf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        arr[i] /= nf;
}

// Fixed-order FP64 block reduction: per-thread Kahan accumulation, then a tree.
__device__ __forceinline__ void kahan_add(double& s, double& c, double x) {
    const double y = x - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
}
__device__ __forceinline__ void block_store_sum(double s, double* out) {
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// kernel_calc_fen (eom.hpp:111-128): f = 1/2 psi (lpsi - psi + 1/2 psi^3), written
// into lpsi like the reference; block partial sums in FP64.
template <typename T>
__global__ void __launch_bounds__(256) k_calc_fen(const T* __restrict__ psi, T* __restrict__ lpsi, int64_t n,
                                                  double* __restrict__ partial) {
    double s = 0.0, c = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T p = psi[i];
        const T f = T(0.5) * p * (lpsi[i] - p + T(0.5) * p * p * p);
        lpsi[i] = f;
        kahan_add(s, c, (double)f);
    }
    block_store_sum(s, partial);
}

// sum over the half spectrum of w_k |psi^_k|^2 (L^_k - 1), w_k = 2 for 0 < i0 < nx/2
// (Parseval: sum_x psi (L-1) psi = (1/N) sum_k |psi^_k|^2 (L^_k - 1) over the full grid).
template <typename T>
__global__ void __launch_bounds__(256) k_fen_spectral(const cx<T>* __restrict__ kpsi, int nx, int ny, int nz, double eps,
                                                      double lx, double ly, double lz, double* __restrict__ partial) {
    const int nxh = nx / 2 + 1;
    const int64_t total = (int64_t)nxh * ny * nz;
    double s = 0.0, c = 0.0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % nxh);
        const int64_t r = idx / nxh;
        const int i1 = (int)(r % ny), i2 = (int)(r / ny);
        const double k0 = kwave<double>(i0, nx, lx), k1 = kwave<double>(i1, ny, ly), k2 = kwave<double>(i2, nz, lz);
        const double k2s = k0 * k0 + k1 * k1 + k2 * k2;
        const double lm1 = (1.0 - eps) - 2.0 * k2s + k2s * k2s;
        const double w = (i0 == 0 || (((nx & 1) == 0) && i0 == nx / 2)) ? 1.0 : 2.0;
        const cx<T> p = kpsi[idx];
        const double a2 = (double)p.x * p.x + (double)p.y * p.y;
        kahan_add(s, c, w * a2 * lm1);
    }
    block_store_sum(s, partial);
}

// sum_x (mul * v)^4 over a real field
template <typename T>
__global__ void __launch_bounds__(256) k_quartic(const T* __restrict__ v, int64_t n, double mul,
                                                 double* __restrict__ partial) {
    double s = 0.0, c = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p = (double)v[i] * mul;
        const double p2 = p * p;
        kahan_add(s, c, p2 * p2);
    }
    block_store_sum(s, partial);
}

__global__ void k_reduce_final(const double* __restrict__ partial, int nb, double scale, double* out) {
    __shared__ double sh[256];
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) kahan_add(s, c, partial[i]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0] * scale;
}

template <typename T>
__global__ void k_noise_kspace(cx<T>* __restrict__ arr, int nx, int ny, int nz, uint64_t seed, uint64_t counter) {
    const int nxh = nx / 2 + 1;
    const int64_t total = (int64_t)nxh * ny * nz;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % nxh);
        const int64_t r = idx / nxh;
        arr[idx] = kspace_noise<T>(i0, (int)(r % ny), (int)(r / ny), nx, ny, nz, seed, counter);
    }
}

template <typename T>
__global__ void k_noise_real(T* __restrict__ arr, int64_t n, T sigma, uint64_t seed, uint64_t counter) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T g1, g2;
        philox_normal2<T>((uint64_t)i, seed, counter, kRealDomain, g1, g2);
        arr[i] = g1 * sigma;
    }
}

template <typename T>
__global__ void k_k0_save(const cx<T>* __restrict__ kpsi, double2* k0) {
    *k0 = make_double2((double)kpsi[0].x, (double)kpsi[0].y);
}

template <typename T>
__global__ void k_k0_restore(cx<T>* __restrict__ kpsi, const double2* k0) {
    kpsi[0] = mkc<T>((T)k0->x, (T)k0->y);
}

__global__ void k_counter(unsigned long long* ctr, int n, unsigned long long value, int set) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (set) ctr[i] = value;
        else ctr[i] += 1ull;
    }
}

}  // namespace

cudaError_t launch_k0_restore(const pfc_ctx* c, void* kpsi) {
    if (c->dtype == PFC_F64) k_k0_restore<double><<<1, 1, 0, c->stream>>>((cx<double>*)kpsi, c->k0);
    else k_k0_restore<float><<<1, 1, 0, c->stream>>>((cx<float>*)kpsi, c->k0);
    return cudaGetLastError();
}

cudaError_t launch_counter(cudaStream_t st, unsigned long long* ctr, unsigned long long value, int set, int n) {
    k_counter<<<1, 128, 0, st>>>(ctr, n, value, set);
    return cudaGetLastError();
}

cudaError_t launch_update_eom(const pfc_ctx* c, void* kpsi, const void* knl, const void* knoise, double namp,
                              double dt, double eps, double lx, double ly, double lz, int with_fen, double C) {
    const int g = grid_for(c->n_cmpl, 256);
    if (c->dtype == PFC_F64) {
        // reference: namp *= sqrtf(nx*ny*nz)  (eom.hpp:62)
        const double ne = namp * (double)sqrtf((float)(c->nx * c->ny * c->nz));
        k_update_eom<double><<<g, 256, 0, c->stream>>>((cx<double>*)kpsi, (const cx<double>*)knl, (cx<double>*)knoise,
                                                        c->nx, c->ny, c->nz, ne, dt, eps, lx, ly, lz, with_fen, C);
    } else {
        const float ne = (float)namp * sqrtf((float)(c->nx * c->ny * c->nz));
        k_update_eom<float><<<g, 256, 0, c->stream>>>((cx<float>*)kpsi, (const cx<float>*)knl, (cx<float>*)knoise,
                                                       c->nx, c->ny, c->nz, ne, (float)dt, (float)eps, (float)lx,
                                                       (float)ly, (float)lz, with_fen, (float)C);
    }
    return cudaGetLastError();
}

cudaError_t launch_psi3(const pfc_ctx* c, void* arr, const void* pot, double mu, int norm, double C) {
    const int64_t n = (int64_t)c->n_real;
    const int g = grid_for(c->n_real, 512);
    if (c->dtype == PFC_F64) {
        const double nf = norm ? 1.0 / (double)n : 1.0;
        k_psi3<double><<<g, 512, 0, c->stream>>>((double*)arr, (const double*)pot, n, nf, mu, C);
    } else {
        // reference: Float nf = 1; nf /= elems  (psi3_split.hpp:18-20)
        float nf = 1.f;
        if (norm) nf /= (float)n;
        k_psi3<float><<<g, 512, 0, c->stream>>>((float*)arr, (const float*)pot, n, nf, (float)mu, (float)C);
    }
    return cudaGetLastError();
}

cudaError_t launch_norm(const pfc_ctx* c, void* arr) {
    const int64_t n = (int64_t)c->n_real;
    const int g = grid_for(c->n_real, 512);
    if (c->dtype == PFC_F64) k_norm<double><<<g, 512, 0, c->stream>>>((double*)arr, n, (double)n);
    else k_norm<float><<<g, 512, 0, c->stream>>>((float*)arr, n, (float)n);
    return cudaGetLastError();
}

cudaError_t launch_reduce_final(const pfc_ctx* c, int slot, double scale) {
    k_reduce_final<<<1, 256, 0, c->stream>>>(c->red, kRedBlocks, scale, c->red + kRedBlocks + slot);
    return cudaGetLastError();
}

cudaError_t launch_calc_fen(const pfc_ctx* c, const void* psi, void* lpsi, double scale) {
    const int64_t n = (int64_t)c->n_real;
    if (c->dtype == PFC_F64) k_calc_fen<double><<<kRedBlocks, 256, 0, c->stream>>>((const double*)psi, (double*)lpsi, n, c->red);
    else k_calc_fen<float><<<kRedBlocks, 256, 0, c->stream>>>((const float*)psi, (float*)lpsi, n, c->red);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    return launch_reduce_final(c, 0, scale);
}

cudaError_t launch_fen_spectral(const pfc_ctx* c, const void* kpsi, double eps, double lx, double ly, double lz) {
    if (c->dtype == PFC_F64)
        k_fen_spectral<double><<<kRedBlocks, 256, 0, c->stream>>>((const cx<double>*)kpsi, c->nx, c->ny, c->nz, eps,
                                                                   lx, ly, lz, c->red);
    else
        k_fen_spectral<float><<<kRedBlocks, 256, 0, c->stream>>>((const cx<float>*)kpsi, c->nx, c->ny, c->nz, eps, lx,
                                                                  ly, lz, c->red);
    return cudaGetLastError();
}

cudaError_t launch_quartic_sum(const pfc_ctx* c, const void* v, double mul) {
    const int64_t n = (int64_t)c->n_real;
    if (c->dtype == PFC_F64) k_quartic<double><<<kRedBlocks, 256, 0, c->stream>>>((const double*)v, n, mul, c->red);
    else k_quartic<float><<<kRedBlocks, 256, 0, c->stream>>>((const float*)v, n, mul, c->red);
    return cudaGetLastError();
}

cudaError_t launch_noise_kspace(const pfc_ctx* c, void* arr, uint64_t seed, uint64_t counter) {
    const int g = grid_for(c->n_cmpl, 256);
    if (c->dtype == PFC_F64)
        k_noise_kspace<double><<<g, 256, 0, c->stream>>>((cx<double>*)arr, c->nx, c->ny, c->nz, seed, counter);
    else
        k_noise_kspace<float><<<g, 256, 0, c->stream>>>((cx<float>*)arr, c->nx, c->ny, c->nz, seed, counter);
    return cudaGetLastError();
}

cudaError_t launch_noise_real(const pfc_ctx* c, void* arr, double sigma, uint64_t seed, uint64_t counter) {
    const int64_t n = (int64_t)c->n_real;
    const int g = grid_for(c->n_real, 256);
    if (c->dtype == PFC_F64) k_noise_real<double><<<g, 256, 0, c->stream>>>((double*)arr, n, sigma, seed, counter);
    else k_noise_real<float><<<g, 256, 0, c->stream>>>((float*)arr, n, (float)sigma, seed, counter);
    return cudaGetLastError();
}

cudaError_t launch_k0_save(const pfc_ctx* c, const void* kpsi) {
    if (c->dtype == PFC_F64) k_k0_save<double><<<1, 1, 0, c->stream>>>((const cx<double>*)kpsi, c->k0);
    else k_k0_save<float><<<1, 1, 0, c->stream>>>((const cx<float>*)kpsi, c->k0);
    return cudaGetLastError();
}

}  // namespace pfc
