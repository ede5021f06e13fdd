// Fused xy-plane kernel of the stepper (FP32): one pass over the carried state.
//
// The stepper carries A = IFFT_z(psi^)/nz (k-space in x and y, real space in z).  For
// one z-plane this kernel computes B = FFT_xy( (psi)^3 - C psi - mu ) with psi =
// IFFT_xy(A) / (nx ny): inverse y FFT, inverse real x FFT, the cubic term, forward
// real x FFT, forward y FFT -- reading the plane once and writing it once (2 x S bytes
// per step instead of 6 x S for three separate passes).
//
// A plane of nx/2 packed complex columns (the kx = 0 and kx = nx/2 columns, whose
// y-transforms are real, ride together as one complex column) by ny rows is split
// over a thread-block cluster of K CTAs: CTA c holds columns [c CPC, (c+1) CPC) for the
// y transforms and rows [c RPC, (c+1) RPC) for the x transforms.  The two transposes
// between them go through distributed shared memory: every thread stores its values
// straight into the owning CTA's shared memory (st.shared::cluster), bracketed by
// cluster barriers.  Data stay in registers (E complex per thread) through each
// four-step FFT; shared memory holds only the transposes.
#include <cooperative_groups.h>
#include <cstdlib>
#include "pfc_ctx.h"
#include "regfft.cuh"

namespace cg = cooperative_groups;

namespace pfc {
namespace {

constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int NX_, int NY_, int K_, int T_>
struct PlaneCfg {
    static constexpr int NX = NX_, NY = NY_, K = K_, T = T_;
    static constexpr int PX = NX / 2, NXH = NX / 2 + 1;
    static constexpr int CPC = PX / K, RPC = NY / K;
    static constexpr int E = PX * NY / (K * T);
    static constexpr int PC = NY / E, PR = PX / E;
    static constexpr int UC = E / PC, UR = E / PR;
    static constexpr int LDR = PX + 1;   // row-major rows of the x phase (odd: conflict-free columns)
    static constexpr int LDC = CPC + 1;  // rows of the y phase receive buffer
    static constexpr int BUF = cmax(T * E, cmax(RPC * LDR, NY * LDC));
    static constexpr int TWN = NY + PX + PX + 1;  // W_NY^m, W_PX^m, W_NX^k (k <= PX)
    static constexpr size_t SMEM = (size_t)(BUF + TWN) * sizeof(float2);
    static constexpr int MINB = T <= 256 ? 2 : 1;  // CTAs per SM the register budget allows
    static_assert(CPC * PC == T && RPC * PR == T, "thread layout");
    static_assert(E % PC == 0 && E % PR == 0, "four-step needs E >= P");
    static_assert(CPC >= 16 && RPC >= 32 && 32 % CPC == 0, "a warp spans 32 rows or 32/CPC t-values of CPC columns");
};

template <class Cfg>
__global__ void __launch_bounds__(Cfg::T, Cfg::MINB)
    k_plane_xy(const float2* __restrict__ A, float2* __restrict__ B, const float* __restrict__ pot,
               const float2* __restrict__ twg, float mul, float Cc, float mu) {
    constexpr int NX = Cfg::NX, NY = Cfg::NY, K = Cfg::K, T = Cfg::T, PX = Cfg::PX, NXH = Cfg::NXH;
    constexpr int CPC = Cfg::CPC, RPC = Cfg::RPC, E = Cfg::E, PC = Cfg::PC, PR = Cfg::PR;
    constexpr int UC = Cfg::UC, UR = Cfg::UR, LDR = Cfg::LDR, LDC = Cfg::LDC;
    extern __shared__ __align__(16) float2 sm[];
    float2* buf = sm;
    float2* twY = sm + Cfg::BUF;
    float2* twX = twY + NY;
    float2* twP = twX + PX;
    const int tid = threadIdx.x;
    for (int i = tid; i < Cfg::TWN; i += T) twY[i] = twg[i];

    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int z = blockIdx.x / K;
    const int64_t plane = (int64_t)z * NY * NXH;

    // ---- phase 1: inverse y FFT of CPC packed columns ------------------------------------
    const int c = tid % CPC, t = tid / CPC, col = rank * CPC + c;
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const float2* row = A + plane + (int64_t)(t + PC * j) * NXH;
        float2 a = row[col];
        if (col == 0) {
            const float2 b = row[PX];
            a = make_float2(a.x - b.y, a.y + b.x);  // A(0, y) + i A(nx/2, y)
        }
        v[j] = a;
    }
    __syncthreads();
    fft_d1_to_d2<NY, E, CPC, 1>(v, t, c, buf, twY);
    cl.sync();
#pragma unroll
    for (int u = 0; u < UC; ++u)
#pragma unroll
        for (int k2 = 0; k2 < PC; ++k2) {
            const int y = (t * UC + u) + E * k2;
            const int dst = y / RPC;
            dsmem_st(dsmem_addr(buf + (y - dst * RPC) * LDR + col, dst), v[u * PC + k2]);
        }
    cl.sync();

    // ---- phase 2: inverse real x FFT, cubic term, forward real x FFT of RPC rows --------
    const int r = tid % RPC, tr = tid / RPC, yg = rank * RPC + r;
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int k = tr + PR * j;
        const float2 xk = buf[r * LDR + k];
        v[j] = (k == 0) ? make_float2(xk.x + xk.y, xk.x - xk.y) : c2r_pre_f(xk, buf[r * LDR + PX - k], twP[k]);
    }
    fft_d1_to_d2<PX, E, RPC, 1>(v, tr, r, buf, twX);
    const int64_t prow = ((int64_t)z * NY + yg) * NX;
#pragma unroll
    for (int u = 0; u < UR; ++u)
#pragma unroll
        for (int k2 = 0; k2 < PR; ++k2) {
            const int n = (tr * UR + u) + E * k2;
            const float2 x = v[u * PR + k2];
            const float a = x.x * mul, b = x.y * mul;
            float2 o = make_float2(a * a * a - Cc * a - mu, b * b * b - Cc * b - mu);
            if (pot) {
                const float2 pp = *reinterpret_cast<const float2*>(pot + prow + 2 * n);
                o.x += pp.x;
                o.y += pp.y;
            }
            v[u * PR + k2] = o;
        }
    fft_d2_to_d1<PX, E, RPC, -1>(v, tr, r, buf, twX);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) buf[r * LDR + tr + PR * j] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int k = tr + PR * j;
        const float2 yk = v[j];
        v[j] = (k == 0) ? make_float2(yk.x + yk.y, yk.x - yk.y)  // X[0], X[nx/2], both real
                        : r2c_post_f(yk, buf[r * LDR + PX - k], twP[k]);
    }
    cl.sync();
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int k = tr + PR * j;
        const int dst = k / CPC;
        dsmem_st(dsmem_addr(buf + yg * LDC + (k - dst * CPC), dst), v[j]);
    }
    cl.sync();

    // ---- phase 3: forward y FFT of CPC packed columns -------------------------------------
#pragma unroll
    for (int u = 0; u < UC; ++u)
#pragma unroll
        for (int n2 = 0; n2 < PC; ++n2) v[u * PC + n2] = buf[((t * UC + u) + E * n2) * LDC + c];
    fft_d2_to_d1<NY, E, CPC, -1>(v, t, c, buf, twY);
    if (rank == 0) {  // unpack column 0 into kx = 0 and kx = nx/2 (Hermitian in ky)
        __syncthreads();
        if (c == 0)
#pragma unroll
            for (int j = 0; j < E; ++j) buf[t + PC * j] = v[j];
        __syncthreads();
        if (c == 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int ky = t + PC * j;
                const float2 zz = v[j], zm = buf[(NY - ky) & (NY - 1)];
                float2* row = B + plane + (int64_t)ky * NXH;
                row[0] = make_float2(0.5f * (zz.x + zm.x), 0.5f * (zz.y - zm.y));
                row[PX] = make_float2(0.5f * (zz.y + zm.y), -0.5f * (zz.x - zm.x));
            }
        }
    }
    if (col != 0) {
#pragma unroll
        for (int j = 0; j < E; ++j) B[plane + (int64_t)(t + PC * j) * NXH + col] = v[j];
    }
}

// Variants: id -> (NX, NY, K, T).  512^2 planes: 16-CTA clusters of 256 threads with
// 76 KB of shared memory each, so two CTAs share an SM (variant 5 keeps 8 CTAs of 512).
using V1 = PlaneCfg<512, 512, 16, 256>;
using V5 = PlaneCfg<512, 512, 8, 512>;
using V2 = PlaneCfg<256, 256, 4, 256>;
using V3 = PlaneCfg<128, 128, 2, 256>;
using V4 = PlaneCfg<64, 64, 1, 128>;

template <class Cfg>
cudaError_t set_attr() {
    cudaError_t e = cudaFuncSetAttribute(k_plane_xy<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
    if (e) return e;
    if (Cfg::K > 8) e = cudaFuncSetAttribute(k_plane_xy<Cfg>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

template <class Cfg>
cudaError_t launch(const pfc_ctx* c, const void* A, void* B, const void* pot, double mul, double C, double mu) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(Cfg::K * c->nz);
    cfg.blockDim = dim3(Cfg::T);
    cfg.dynamicSmemBytes = Cfg::SMEM;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = Cfg::K;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->plane_tw_off;
    return cudaLaunchKernelEx(&cfg, k_plane_xy<Cfg>, (const float2*)A, (float2*)B, (const float*)pot, tw, (float)mul,
                              (float)C, (float)mu);
}

}  // namespace

int fused_xy_variant(int nx, int ny, int dtype) {
    if (dtype != PFC_F32) return 0;
    if (nx == 512 && ny == 512) {
        const char* f = getenv("PFC_PLANE_VARIANT");
        return (f && atoi(f) == 5) ? 5 : 1;
    }
    if (nx == 256 && ny == 256) return 2;
    if (nx == 128 && ny == 128) return 3;
    if (nx == 64 && ny == 64) return 4;
    return 0;
}

cudaError_t set_fused_attributes(const pfc_ctx* c) {
    switch (c->fused_xy) {
        case 1: return set_attr<V1>();
        case 2: return set_attr<V2>();
        case 3: return set_attr<V3>();
        case 4: return set_attr<V4>();
        case 5: return set_attr<V5>();
    }
    return cudaSuccess;
}

cudaError_t launch_fused_xy(const pfc_ctx* c, const void* A, void* B, const void* pot, double mul, double C,
                            double mu) {
    switch (c->fused_xy) {
        case 1: return launch<V1>(c, A, B, pot, mul, C, mu);
        case 2: return launch<V2>(c, A, B, pot, mul, C, mu);
        case 3: return launch<V3>(c, A, B, pot, mul, C, mu);
        case 4: return launch<V4>(c, A, B, pot, mul, C, mu);
        case 5: return launch<V5>(c, A, B, pot, mul, C, mu);
    }
    return cudaErrorNotSupported;
}

}  // namespace pfc
