// The reference's other per-mode propagators, as mirror kernels of its arithmetic
// (single-precision expf/sqrtf where the reference calls them, even for double fields):
//
//  k_init_eom_op / k_update_eom_exp   conserved exponential time differencing
//                                     (cuda/kernels/eom-exp.hpp:3-60)
//  k_update_el                        non-conserved semi-implicit relaxation with the
//                                     largest mode change (cuda/kernels/el.hpp:3-45), and
//                                     its exponential form (cuda/kernels/el-exp.hpp:17-60)
//  k_init_el_op                       the operator of that form (el-exp.hpp:3-15)
//  k_update_eom_py                    conserved update with the polynomial kernel
//                                     (cuda/kernels/eom.hpp:143-180)
//  k_update_eom_hpfcnoise             2D conserved update with the anisotropic noise of
//                                     three fields (cuda/kernels/eom.hpp:16-58)
//
// The largest change max_k |psi^'_k - psi^_k| of the relaxation kernels is reduced with
// a block maximum and an atomicMax on the bits of a non-negative float (order-free,
// so deterministic); the reference reduces per block on the device and then on the host.
#include "pfc_ctx.h"

namespace pfc {
namespace {

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    const size_t cap = 148 * 16;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

template <typename T> __device__ __forceinline__ T f_sqrt(T x) { return (T)sqrtf((float)x); }
template <typename T> __device__ __forceinline__ T f_exp(T x) { return (T)expf((float)x); }

struct Modes {
    int nx, ny, nz;
    __device__ __forceinline__ int64_t total() const { return (int64_t)(nx / 2 + 1) * ny * nz; }
    __device__ __forceinline__ void at(int64_t idx, int& i0, int& i1, int& i2) const {
        const int nxh = nx / 2 + 1;
        i0 = (int)(idx % nxh);
        const int64_t r = idx / nxh;
        i1 = (int)(r % ny);
        i2 = (int)(r / ny);
    }
};

// dop = (-k^2, k^4) of L_L2 (common.hpp:17-22) with K (common.hpp:27-28)
template <typename T>
__device__ __forceinline__ void dop_at(const Modes& m, int i0, int i1, int i2, T lx, T ly, T lz, T& dx, T& dy,
                                       T* k0 = nullptr, T* k1 = nullptr) {
    const T a = kwave<T>(i0, m.nx, lx), b = kwave<T>(i1, m.ny, ly), c = kwave<T>(i2, m.nz, lz);
    dx = -a * a - b * b - c * c;
    dy = dx * dx;
    if (k0) *k0 = a;
    if (k1) *k1 = b;
}

#define PFC_MODE_LOOP(m)                                                                                 \
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (m).total();              \
         idx += (int64_t)gridDim.x * blockDim.x)

template <typename T>
__global__ void k_init_eom_op(cx<T>* kop, Modes m, T dt, T eps, T lx, T ly, T lz) {
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        T dx, dy;
        dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy);
        const T lin = -dx * ((T(2) - eps) + T(2) * dx + dy);
        const T e = f_exp<T>(-lin * dt);
        const T second = (e - T(1)) / lin;  // 0/0 at k = 0
        kop[idx] = mkc<T>(e, second == second ? second : -dt);
    }
}

template <typename T>
__global__ void k_update_eom_exp(const cx<T>* __restrict__ kop, cx<T>* kpsi, const cx<T>* __restrict__ knl,
                                 cx<T>* knoise, Modes m, T namp_eff, T eps, T lx, T ly, T lz, int with_fen) {
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        T dx, dy;
        dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy);
        const T k = f_sqrt<T>(-dx);
        const cx<T> p = kpsi[idx], q = knl[idx], o = kop[idx];
        const cx<T> w = knoise ? knoise[idx] : mkc<T>(T(0), T(0));
        kpsi[idx] = mkc<T>(p.x * o.x - dx * q.x * o.y - namp_eff * k * w.x * o.y,
                           p.y * o.x - dx * q.y * o.y - namp_eff * k * w.y * o.y);
        if (with_fen) {
            const T lk = (T(2) - eps) + T(2) * dx + dy;
            knoise[idx] = mkc<T>(lk * p.x, lk * p.y);
        }
    }
}

__device__ __forceinline__ void block_max_to(float v, float* out) {
    __shared__ float sh[256];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    // non-negative floats order like their bit patterns
    if (threadIdx.x == 0) atomicMax(reinterpret_cast<unsigned int*>(out), __float_as_uint(sh[0]));
}

// kop == nullptr: el.hpp (semi-implicit); otherwise el-exp.hpp (kop given)
template <typename T>
__global__ void __launch_bounds__(256) k_update_el(const cx<T>* __restrict__ kop, cx<T>* kpsi,
                                                   const cx<T>* __restrict__ knl, Modes m, T dt, T eps, T lx, T ly,
                                                   T lz, float* max_change) {
    float mx = 0.f;
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        const cx<T> p = kpsi[idx], q = knl[idx];
        cx<T> r;
        if (kop) {
            const cx<T> o = kop[idx];
            r = mkc<T>(p.x * o.x + q.x * o.y, p.y * o.x + q.y * o.y);
        } else {
            T dx, dy;
            dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy);
            const T denom = T(1) + dt * ((T(2) - eps) + T(2) * dx + dy);
            r = mkc<T>((p.x - dt * q.x) / denom, (p.y - dt * q.y) / denom);
        }
        kpsi[idx] = r;
        const T ex = p.x - r.x, ey = p.y - r.y;
        mx = fmaxf(mx, (float)sqrt(ex * ex + ey * ey));
    }
    block_max_to(mx, max_change);
}

template <typename T>
__global__ void k_init_el_op(cx<T>* kop, Modes m, T dt, T eps, T lx, T ly, T lz) {
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        T dx, dy;
        dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy);
        const T lin = (T(2) - eps) + T(2) * dx + dy;
        const T e = f_exp<T>(-lin * dt);
        kop[idx] = mkc<T>(e, (e - T(1)) / lin);
    }
}

template <typename T>
__global__ void k_update_eom_py(cx<T>* kpsi, const cx<T>* __restrict__ knl, const cx<T>* __restrict__ knoise,
                                Modes m, T namp_eff, T dt, T eps, T lx, T ly, T lz) {
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        T dx, dy;
        dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy);
        const T k2 = -dx;
        const T k = f_sqrt<T>(k2);
        const T denom = T(1) - dt * dx * (T(1) - eps - py_poly<T>(k2));
        const cx<T> p = kpsi[idx], q = knl[idx];
        const cx<T> w = knoise ? knoise[idx] : mkc<T>(T(0), T(0));
        kpsi[idx] = mkc<T>((p.x + dt * dx * q.x + dt * namp_eff * k * w.x) / denom,
                           (p.y + dt * dx * q.y + dt * namp_eff * k * w.y) / denom);
    }
}

template <typename T>
__global__ void k_update_eom_hpfcnoise(cx<T>* kpsi, const cx<T>* __restrict__ knl, const cx<T>* __restrict__ n1,
                                       const cx<T>* __restrict__ n2, const cx<T>* __restrict__ n3, Modes m,
                                       T namp_eff, T dt, T eps, T lx, T ly, T lz) {
    const T kappa = T(4) / T(3);
    const T c2 = f_sqrt<T>(T(1) + kappa / T(2) + f_sqrt<T>(T(1) + kappa));
    const T c1 = kappa / c2 / T(2);
    PFC_MODE_LOOP(m) {
        int i0, i1, i2;
        m.at(idx, i0, i1, i2);
        T dx, dy, k0, k1;
        dop_at<T>(m, i0, i1, i2, lx, ly, lz, dx, dy, &k0, &k1);
        const T k = f_sqrt<T>(-dx);
        const T denom = T(1) - dt * ((T(2) - eps) * dx + T(2) * dy + dx * dy);
        const cx<T> a = n1[idx], b = n2[idx], c = n3[idx];
        const T fa = c1 * k0 * k0 + c2 * k1 * k1, fb = c2 * k0 * k0 + c1 * k1 * k1, fc = T(2) * k0 * k1;
        T nx_ = fa * a.x + fb * b.x + fc * c.x;
        T ny_ = fa * a.y + fb * b.y + fc * c.y;
        if (!(k <= T(0.25))) nx_ = ny_ = T(0);
        const cx<T> p = kpsi[idx], q = knl[idx];
        kpsi[idx] = mkc<T>((p.x + dt * dx * q.x + dt * namp_eff * nx_) / denom,
                           (p.y + dt * dx * q.y + dt * namp_eff * ny_) / denom);
    }
}

Modes modes(const pfc_ctx* c) { return Modes{c->nx, c->ny, c->nz}; }

// the reference's namp *= sqrtf(nx*ny*nz), in the field's precision
double namp_scaled(const pfc_ctx* c, double namp) {
    const float s = sqrtf((float)(c->nx * c->ny * c->nz));
    return c->dtype == PFC_F64 ? namp * (double)s : (double)((float)namp * s);
}

}  // namespace

#define PFC_DISPATCH(c, KERNEL, grid, block, shmem, ...)                                                   \
    do {                                                                                                    \
        if ((c)->dtype == PFC_F64) {                                                                       \
            using T = double;                                                                              \
            KERNEL<T><<<grid, block, shmem, (c)->stream>>>(__VA_ARGS__);                                   \
        } else {                                                                                            \
            using T = float;                                                                               \
            KERNEL<T><<<grid, block, shmem, (c)->stream>>>(__VA_ARGS__);                                   \
        }                                                                                                   \
    } while (0)

cudaError_t launch_init_eom_op(const pfc_ctx* c, void* kop, double dt, double eps, double lx, double ly, double lz) {
    PFC_DISPATCH(c, k_init_eom_op, grid_for(c->n_cmpl, 256), 256, 0, (cx<T>*)kop, modes(c), (T)dt, (T)eps, (T)lx,
                 (T)ly, (T)lz);
    return cudaGetLastError();
}

cudaError_t launch_update_eom_exp(const pfc_ctx* c, const void* kop, void* kpsi, const void* knl, void* knoise,
                                  double namp, double eps, double lx, double ly, double lz, int with_fen) {
    const double ne = namp_scaled(c, namp);
    PFC_DISPATCH(c, k_update_eom_exp, grid_for(c->n_cmpl, 256), 256, 0, (const cx<T>*)kop, (cx<T>*)kpsi,
                 (const cx<T>*)knl, (cx<T>*)knoise, modes(c), (T)ne, (T)eps, (T)lx, (T)ly, (T)lz, with_fen);
    return cudaGetLastError();
}

cudaError_t launch_init_el_op(const pfc_ctx* c, void* kop, double dt, double eps, double lx, double ly, double lz) {
    PFC_DISPATCH(c, k_init_el_op, grid_for(c->n_cmpl, 256), 256, 0, (cx<T>*)kop, modes(c), (T)dt, (T)eps, (T)lx,
                 (T)ly, (T)lz);
    return cudaGetLastError();
}

// the largest change lands in c->red (as float bits) and is copied to *max_change
cudaError_t launch_update_el(const pfc_ctx* c, const void* kop, void* kpsi, const void* knl, double dt, double eps,
                             double lx, double ly, double lz, double* max_change) {
    float* slot = reinterpret_cast<float*>(c->red + kRedBlocks + 3);
    cudaError_t e = cudaMemsetAsync(slot, 0, sizeof(float), c->stream);
    if (e) return e;
    PFC_DISPATCH(c, k_update_el, kRedBlocks, 256, 0, (const cx<T>*)kop, (cx<T>*)kpsi, (const cx<T>*)knl, modes(c),
                 (T)dt, (T)eps, (T)lx, (T)ly, (T)lz, slot);
    if ((e = cudaGetLastError())) return e;
    float h = 0.f;
    if ((e = cudaMemcpyAsync(&h, slot, sizeof(float), cudaMemcpyDeviceToHost, c->stream))) return e;
    if ((e = cudaStreamSynchronize(c->stream))) return e;
    *max_change = (double)h;
    return cudaSuccess;
}

cudaError_t launch_update_eom_py(const pfc_ctx* c, void* kpsi, const void* knl, const void* knoise, double namp,
                                 double dt, double eps, double lx, double ly, double lz) {
    const double ne = namp_scaled(c, namp);
    PFC_DISPATCH(c, k_update_eom_py, grid_for(c->n_cmpl, 256), 256, 0, (cx<T>*)kpsi, (const cx<T>*)knl,
                 (const cx<T>*)knoise, modes(c), (T)ne, (T)dt, (T)eps, (T)lx, (T)ly, (T)lz);
    return cudaGetLastError();
}

cudaError_t launch_update_eom_hpfcnoise(const pfc_ctx* c, void* kpsi, const void* knl, const void* n1, const void* n2,
                                        const void* n3, double namp, double dt, double eps, double lx, double ly,
                                        double lz) {
    const double ne = namp_scaled(c, namp);
    PFC_DISPATCH(c, k_update_eom_hpfcnoise, grid_for(c->n_cmpl, 256), 256, 0, (cx<T>*)kpsi, (const cx<T>*)knl,
                 (const cx<T>*)n1, (const cx<T>*)n2, (const cx<T>*)n3, modes(c), (T)ne, (T)dt, (T)eps, (T)lx, (T)ly,
                 (T)lz);
    return cudaGetLastError();
}

#undef PFC_DISPATCH

}  // namespace pfc
