// The stepper's z pass for FP32 grids with nz in {64, 128, 256, 512}: register-resident
// four-step FFTs along z for a tile of TX consecutive kx columns at one ky.
//
// The first half of the CTA transforms the carried state A (psi^ = FFT_z(A)), the second
// half the nonlinear term B (N^ = FFT_z(B)), concurrently, each behind its own named
// barrier.  N^ is handed over through shared memory; the first half then applies the
// semi-implicit update of eom.hpp:60-72 (stabilisation C, conserved Philox noise, the
// FP64 k = 0 mode, non-finite watchdog) and transforms back, A' = IFFT_z(psi^')/nz, or
// stores psi^' itself on the last step.  The kx = nx/2 column is left to the general
// z kernel (one narrow launch).
#include "pfc_ctx.h"
#include "regfft.cuh"

namespace pfc {
namespace {

template <int NZ_, int E_, int TX_>
struct ZCfg {
    static constexpr int NZ = NZ_, E = E_, TX = TX_;
    static constexpr int P = NZ / E, U = E / P;
    static constexpr int TH = TX * P;  // threads per field
    static constexpr int T = 2 * TH;
    static constexpr int PADG = TX / U;  // exchange padding: the 32/TX t-groups of a warp hit distinct banks
    static constexpr int REG = E * (P * TX + PADG);
    static constexpr size_t SMEM = (size_t)(2 * REG + NZ) * sizeof(float2);
    static_assert(TH % 32 == 0 && U * P == E && TX % U == 0 && 32 % TX == 0, "shape");
};

struct ZArgsF {
    float dt, eps, C, namp_eff, ckx, cky, ckz;  // ck = 2 pi / L per axis
    uint64_t seed, counter;
    int use_noise, final_step;
};

template <class Z>
__global__ void __launch_bounds__(Z::T, 2) k_zcol(float2* A, const float2* __restrict__ B, int nx, int ny, ZArgsF a,
                                                   const double2* __restrict__ k0, int* flag,
                                                   const float2* __restrict__ twg) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, U = Z::U, TH = Z::TH;
    extern __shared__ __align__(16) float2 sm[];
    float2* regA = sm;
    float2* regB = sm + Z::REG;
    float2* tw = sm + 2 * Z::REG;
    const int tid = threadIdx.x;
    for (int i = tid; i < NZ; i += Z::T) tw[i] = twg[i];
    const int half = tid / TH;
    const int lt = tid - half * TH;
    const int c = lt % TX, t = lt / TX;
    const int kx = blockIdx.x * TX + c;
    const int ky = blockIdx.y;
    const int nxh = nx / 2 + 1;
    const bool valid = kx < nxh;  // the last tile holds only the kx = nx/2 column
    const int64_t zs = (int64_t)ny * nxh;
    const int64_t base = (int64_t)ky * nxh + kx;
    const float2* src = half ? B : A;
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? src[base + (int64_t)(t + P * j) * zs] : make_float2(0.f, 0.f);
    __syncthreads();
    if (half == 0) {
        fft_d1_to_d2<NZ, E, TX, -1, BarNamed<1, TH>, Z::PADG>(v, t, c, regA, tw);
    } else {
        fft_d1_to_d2<NZ, E, TX, -1, BarNamed<2, TH>, Z::PADG>(v, t, c, regB, tw);
        BarNamed<2, TH>::sync();
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) regB[((t * U + u) + E * k2) * TX + c] = v[u * P + k2];
    }
    __syncthreads();
    if (half != 0) return;

    // wavenumbers K(i) = i' * 2 pi / L (common.hpp:27-28) with 2 pi / L precomputed
    const float k0x = (float)kx * a.ckx;
    const float k1y = (float)(ky < ny / 2 + 1 ? ky : ky - ny) * a.cky;
    const float kxy = k0x * k0x + k1y * k1y;
    const float deps = 1.0f + a.C - a.eps;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) {
            const int kz = (t * U + u) + E * k2;
            float2 psi = v[u * P + k2];
            const float2 nl = regB[kz * TX + c];
            const float k2z = (float)(kz < NZ / 2 + 1 ? kz : kz - NZ) * a.ckz;
            const float dopx = -kxy - k2z * k2z;
            const float dopy = dopx * dopx;
            const float inv = __frcp_rn(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
            if (kx == 0 && ky == 0 && kz == 0) psi = make_float2((float)k0->x, (float)k0->y);
            const float f = a.dt * dopx;
            v[u * P + k2] = make_float2((psi.x + f * nl.x) * inv, (psi.y + f * nl.y) * inv);
        }
    if (a.use_noise) {
        // conserved k-space noise, dt namp sqrt(N) |k| xi / D(k): a compact loop over this
        // thread's modes, staged through its own N^ slots (kept out of the unrolled body)
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) regB[((t * U + u) + E * k2) * TX + c] = v[u * P + k2];
#pragma unroll 1
        for (int m = 0; m < E; ++m) {
            const int kz = (t * U + m / P) + E * (m % P);
            const float k2z = (float)(kz < NZ / 2 + 1 ? kz : kz - NZ) * a.ckz;
            const float dopx = -kxy - k2z * k2z;
            const float dopy = dopx * dopx;
            const float inv = __frcp_rn(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
            const float2 xi = kspace_noise<float>(kx, ky, kz, nx, ny, NZ, a.seed, a.counter);
            const float g = a.dt * a.namp_eff * sqrtf(-dopx) * inv;
            float2 w = regB[kz * TX + c];
            w.x += g * xi.x;
            w.y += g * xi.y;
            regB[kz * TX + c] = w;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) v[u * P + k2] = regB[((t * U + u) + E * k2) * TX + c];
    }
    bool bad = false;
#pragma unroll
    for (int j = 0; j < E; ++j) bad |= !isfinite(v[j].x) || !isfinite(v[j].y);
    if (bad && valid) atomicOr(flag, 1);
    if (a.final_step) {
        if (valid)
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int k2 = 0; k2 < P; ++k2) A[base + (int64_t)((t * U + u) + E * k2) * zs] = v[u * P + k2];
        return;
    }
    fft_d2_to_d1<NZ, E, TX, 1, BarNamed<1, TH>, Z::PADG>(v, t, c, regA, tw);
    const float s = 1.0f / (float)NZ;
    if (valid)
#pragma unroll
        for (int j = 0; j < E; ++j) A[base + (int64_t)(t + P * j) * zs] = make_float2(v[j].x * s, v[j].y * s);
}

using Z512 = ZCfg<512, 32, 8>;
using Z256 = ZCfg<256, 16, 8>;
using Z128 = ZCfg<128, 16, 8>;
using Z64 = ZCfg<64, 8, 8>;

template <class Z>
cudaError_t zattr() {
    return cudaFuncSetAttribute(k_zcol<Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::SMEM);
}

template <class Z>
cudaError_t zlaunch(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& p) {
    const double tp = 6.283185307179586232;
    ZArgsF a{(float)p.dt, (float)p.eps, (float)p.C, (float)p.namp_eff, (float)(tp / p.lx), (float)(tp / p.ly),
             (float)(tp / p.lz), p.seed, p.counter, p.use_noise, p.final_step};
    dim3 grid((c->nxh + Z::TX - 1) / Z::TX, c->ny);
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
    k_zcol<Z><<<grid, Z::T, Z::SMEM, c->stream>>>((float2*)A, (const float2*)B, c->nx, c->ny, a, c->k0, c->flag, tw);
    return cudaGetLastError();
}

}  // namespace

int fused_z_variant(int nx, int nz, int dtype) {
    if (dtype != PFC_F32 || nx < 16 || (nx / 2) % 8 != 0 || nx % 2 != 0) return 0;
    switch (nz) {
        case 512: return 1;
        case 256: return 2;
        case 128: return 3;
        case 64: return 4;
    }
    return 0;
}

cudaError_t set_zcol_attributes(const pfc_ctx* c) {
    switch (c->fused_z) {
        case 1: return zattr<Z512>();
        case 2: return zattr<Z256>();
        case 3: return zattr<Z128>();
        case 4: return zattr<Z64>();
    }
    return cudaSuccess;
}

cudaError_t launch_zcol(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& a) {
    switch (c->fused_z) {
        case 1: return zlaunch<Z512>(c, A, B, a);
        case 2: return zlaunch<Z256>(c, A, B, a);
        case 3: return zlaunch<Z128>(c, A, B, a);
        case 4: return zlaunch<Z64>(c, A, B, a);
    }
    return cudaErrorNotSupported;
}

}  // namespace pfc
