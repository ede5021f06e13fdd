// Reverse mode of the conserved semi-implicit step: no counterpart in mcstar-libs.
//
// Forward map of one step (pfc_step; eom.hpp:60-72 with the stabilisation C):
//   psi^' = D^-1 (psi^ - dt k^2 F[g(psi)]) + D^-1 eta,   g(psi) = psi^3 - C psi - mu,
//   D(k) = 1 + dt k^2 (C - eps + (1 - k^2)^2),   psi = C2R(psi^) / N.
// In real space psi' = M psi - K g(psi) + ..., with M = F^-1 D^-1 F and
// K = F^-1 (dt k^2 / D) F symmetric (D and k^2 are even in k), so the adjoint of a
// real-field sensitivity lam' = dL/dpsi' is
//   lam = M lam' - g'(psi) (K lam'),   g'(psi) = 3 psi^2 - C,
// and eps enters only through D:  d psi^' / d eps = (dt k^2 / D) psi^'  (the noise term
// included), so  dL/deps += <lam', F^-1 (dt k^2 / D) psi^'> = (1/N) sum_k w_k Re(conj(lam^'_k)
// (dt k^2 / D_k) psi^'_k)  (Parseval; w_k = 2 on the interior kx planes of the half
// spectrum).  The structure-factor loss L = sum_k (|psi^_k|^2 / N - s_k)^2 (full
// spectrum) seeds lam_T = (4/N) C2R(r psi^), r_k = |psi^_k|^2 / N - s_k.
//
// All factors are evaluated in FP64; fields keep the context's precision.
#include "pfc_ctx.h"

namespace pfc {
namespace {

struct AdjGeom {
    int nx, ny, nz;
    double lx, ly, lz, dt, eps, C;
};

__device__ __forceinline__ void mode_of(int64_t idx, int nx, int ny, int& i0, int& i1, int& i2) {
    const int nxh = nx / 2 + 1;
    i0 = (int)(idx % nxh);
    const int64_t r = idx / nxh;
    i1 = (int)(r % ny);
    i2 = (int)(r / ny);
}

// 1/D and dt k^2 / D at mode (i0, i1, i2)
__device__ __forceinline__ void prop_factors(const AdjGeom& g, int i0, int i1, int i2, double& inv_d, double& kfac) {
    const double k0 = kwave<double>(i0, g.nx, g.lx), k1 = kwave<double>(i1, g.ny, g.ly), k2 = kwave<double>(i2, g.nz, g.lz);
    const double k2s = k0 * k0 + k1 * k1 + k2 * k2;
    const double om = 1.0 - k2s;
    inv_d = 1.0 / (1.0 + g.dt * k2s * (g.C - g.eps + om * om));
    kfac = g.dt * k2s * inv_d;
}

__device__ __forceinline__ double half_weight(int i0, int nx) {
    return (i0 == 0 || (((nx & 1) == 0) && i0 == nx / 2)) ? 1.0 : 2.0;
}

__device__ __forceinline__ void block_sum(double s, double* out) {
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// out = (1/D) in (mode 0) or (dt k^2 / D) in (mode 1); in may equal out
template <typename T>
__global__ void k_adj_mul(const cx<T>* in, cx<T>* out, AdjGeom g, int mode) {
    const int64_t total = (int64_t)(g.nx / 2 + 1) * g.ny * g.nz;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i0, i1, i2;
        mode_of(idx, g.nx, g.ny, i0, i1, i2);
        double inv_d, kfac;
        prop_factors(g, i0, i1, i2, inv_d, kfac);
        const double f = mode ? kfac : inv_d;
        const cx<T> v = in[idx];
        out[idx] = mkc<T>((T)(f * (double)v.x), (T)(f * (double)v.y));
    }
}

// block partials of sum_k w_k Re(conj(lh_k) (dt k^2 / D_k) p_k)
template <typename T>
__global__ void __launch_bounds__(256) k_adj_eps(const cx<T>* __restrict__ lh, const cx<T>* __restrict__ p, AdjGeom g,
                                                 double* __restrict__ partial) {
    const int64_t total = (int64_t)(g.nx / 2 + 1) * g.ny * g.nz;
    double s = 0.0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i0, i1, i2;
        mode_of(idx, g.nx, g.ny, i0, i1, i2);
        double inv_d, kfac;
        prop_factors(g, i0, i1, i2, inv_d, kfac);
        const cx<T> a = lh[idx], b = p[idx];
        s += half_weight(i0, g.nx) * kfac * ((double)a.x * b.x + (double)a.y * b.y);
    }
    block_sum(s, partial);
}

// lam <- (A - (3 (psi_u / N)^2 - C) B) / N, A (in lam), psi_u and B unnormalised C2R outputs
template <typename T>
__global__ void k_adj_combine(T* __restrict__ lam, const T* __restrict__ psi_u, const T* __restrict__ b, int64_t n,
                              double inv_n, double C) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p = (double)psi_u[i] * inv_n;
        lam[i] = (T)(((double)lam[i] - (3.0 * p * p - C) * (double)b[i]) * inv_n);
    }
}

// r_k = |psi^_k|^2 / N - s_k: partials of sum_k w_k r_k^2, and out_k = (4/N) r_k psi^_k
template <typename T>
__global__ void __launch_bounds__(256) k_sf_loss(const cx<T>* __restrict__ kpsi, const T* __restrict__ s_target,
                                                 cx<T>* __restrict__ out, int nx, int ny, int nz,
                                                 double* __restrict__ partial) {
    const int64_t total = (int64_t)(nx / 2 + 1) * ny * nz;
    const double inv_n = 1.0 / ((double)nx * ny * nz);
    double s = 0.0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i0, i1, i2;
        mode_of(idx, nx, ny, i0, i1, i2);
        const cx<T> v = kpsi[idx];
        const double r = ((double)v.x * v.x + (double)v.y * v.y) * inv_n - (double)s_target[idx];
        s += half_weight(i0, nx) * r * r;
        const double f = 4.0 * inv_n * r;
        out[idx] = mkc<T>((T)(f * (double)v.x), (T)(f * (double)v.y));
    }
    block_sum(s, partial);
}

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    const size_t cap = 148 * 16;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

AdjGeom geom(const pfc_ctx* c, const pfc_step_params* p) {
    return AdjGeom{c->nx, c->ny, c->nz, p->lx, p->ly, p->lz, p->dt, p->eps, p->C};
}

}  // namespace

cudaError_t launch_adj_mul(const pfc_ctx* c, const void* in, void* out, const pfc_step_params* p, int mode) {
    const int g = grid_for(c->n_cmpl, 256);
    if (c->dtype == PFC_F64)
        k_adj_mul<double><<<g, 256, 0, c->stream>>>((const cx<double>*)in, (cx<double>*)out, geom(c, p), mode);
    else
        k_adj_mul<float><<<g, 256, 0, c->stream>>>((const cx<float>*)in, (cx<float>*)out, geom(c, p), mode);
    return cudaGetLastError();
}

cudaError_t launch_adj_eps(const pfc_ctx* c, const void* lam_hat, const void* kpsi_np1, const pfc_step_params* p) {
    if (c->dtype == PFC_F64)
        k_adj_eps<double><<<kRedBlocks, 256, 0, c->stream>>>((const cx<double>*)lam_hat, (const cx<double>*)kpsi_np1,
                                                             geom(c, p), c->red);
    else
        k_adj_eps<float><<<kRedBlocks, 256, 0, c->stream>>>((const cx<float>*)lam_hat, (const cx<float>*)kpsi_np1,
                                                            geom(c, p), c->red);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    return launch_reduce_final(c, 3, 1.0 / ((double)c->nx * c->ny * c->nz));
}

cudaError_t launch_adj_combine(const pfc_ctx* c, void* lam, const void* psi_u, const void* b, double C) {
    const int64_t n = (int64_t)c->n_real;
    const int g = grid_for(c->n_real, 256);
    const double inv_n = 1.0 / (double)n;
    if (c->dtype == PFC_F64)
        k_adj_combine<double><<<g, 256, 0, c->stream>>>((double*)lam, (const double*)psi_u, (const double*)b, n, inv_n,
                                                        C);
    else
        k_adj_combine<float><<<g, 256, 0, c->stream>>>((float*)lam, (const float*)psi_u, (const float*)b, n, inv_n, C);
    return cudaGetLastError();
}

cudaError_t launch_sf_loss(const pfc_ctx* c, const void* kpsi, const void* s_target, void* out) {
    if (c->dtype == PFC_F64)
        k_sf_loss<double><<<kRedBlocks, 256, 0, c->stream>>>((const cx<double>*)kpsi, (const double*)s_target,
                                                             (cx<double>*)out, c->nx, c->ny, c->nz, c->red);
    else
        k_sf_loss<float><<<kRedBlocks, 256, 0, c->stream>>>((const cx<float>*)kpsi, (const float*)s_target,
                                                            (cx<float>*)out, c->nx, c->ny, c->nz, c->red);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    return launch_reduce_final(c, 3, 1.0);
}

}  // namespace pfc
