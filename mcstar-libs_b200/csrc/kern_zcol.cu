// The stepper's z pass for FP32 grids with nz in {64, 128, 256, 512}: register-resident
// four-step FFTs along z on tiles of TX consecutive kx columns at one ky.
//
// Per tile: psi^ = FFT_z(A) (the carried state), N^ = FFT_z(B) (the nonlinear term),
// the semi-implicit update of eom.hpp:60-72 (stabilisation C, conserved Philox noise,
// the FP64 k = 0 mode, non-finite watchdog), then A' = IFFT_z(psi^')/nz -- or psi^'
// itself on the last step.  Half of each CTA transforms A, the other half B.
//
//  k_zcol   one tile per CTA; both halves load and transform concurrently, N^ is
//           handed over through shared memory, then the A half finishes alone.
//  k_zpipe  persistent, one CTA per SM: each half prefetches its next tile with
//           cp.async into a shared staging buffer while it computes the current one,
//           and the B half's forward FFT of tile i+1 overlaps the A half's update and
//           inverse FFT of tile i.  The hand-over of N^ is a producer/consumer pair of
//           named barriers (3: N^ written, 4: slots free again).
#include "pfc_ctx.h"
#include "regfft.cuh"

namespace pfc {
namespace {

struct ZArgsF {
    float dt, eps, C, namp_eff, ckx, cky, ckz;  // ck = 2 pi / L per axis
    uint64_t seed, counter;
    const unsigned long long* dev_counter;      // read instead of counter when set
    int use_noise, final_step;
};

template <int NZ_, int E_, int TX_>
struct ZCfg {
    static constexpr int NZ = NZ_, E = E_, TX = TX_;
    static constexpr int P = NZ / E, U = E / P;
    static constexpr int TH = TX * P;  // threads per field
    static constexpr int T = 2 * TH;
    static constexpr int PADG = TX / U;  // exchange padding: the 32/TX t-groups of a warp hit distinct banks
    static constexpr int REG = E * (P * TX + PADG);
    // N^ slots of the pipelined kernel, skewed by 8 per U modes so that a warp's four
    // t-groups (kz = t U + ...) fall in different banks
    static constexpr int NHS = NZ * TX + (NZ / U) * 8;
    static constexpr int STG = NZ * TX;  // staging of one field tile, [z][c]
    static constexpr size_t SMEM = (size_t)(2 * REG + NZ) * sizeof(float2);
    static constexpr size_t SMEM_PIPE = (size_t)(2 * STG + 2 * REG + NHS + NZ) * sizeof(float2);
    static_assert(TH % 32 == 0 && U * P == E && TX % U == 0 && 32 % TX == 0, "shape");
};

template <class Z> __device__ __forceinline__ int nh_slot(int kz, int c) { return kz * Z::TX + c + (kz / Z::U) * 8; }

// The update of the thread's modes kz = (t U + u) + E k2 of column kx at ky.  nl(kz)
// returns N^; scratch (this thread's own slots kz * TX + c) stages the noise pass, after
// a barrier of the half (Bar) so that no thread of the half still reads its exchange.
template <class Z, class Bar, class NL>
__device__ __forceinline__ void propagate(float2 (&v)[Z::E], NL nl, float2* scratch, int kx, int ky, int t, int c,
                                          int nx, int ny, bool valid, const ZArgsF& a, const double2* k0, int* flag) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, U = Z::U;
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
            const float2 n = nl(kz);
            const float k2z = (float)(kz < NZ / 2 + 1 ? kz : kz - NZ) * a.ckz;
            const float dopx = -kxy - k2z * k2z;
            const float dopy = dopx * dopx;
            const float inv = __frcp_rn(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
            if (kx == 0 && ky == 0 && kz == 0) psi = make_float2((float)k0->x, (float)k0->y);
            const float f = a.dt * dopx;
            v[u * P + k2] = make_float2((psi.x + f * n.x) * inv, (psi.y + f * n.y) * inv);
        }
    if (a.use_noise) {
        // conserved k-space noise, dt namp sqrt(N) |k| xi / D(k): a compact loop over this
        // thread's modes, staged through its own slots (kept out of the unrolled body)
        Bar::sync();
        const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) scratch[((t * U + u) + E * k2) * TX + c] = v[u * P + k2];
#pragma unroll 1
        for (int m = 0; m < E; ++m) {
            const int kz = (t * U + m / P) + E * (m % P);
            const float k2z = (float)(kz < NZ / 2 + 1 ? kz : kz - NZ) * a.ckz;
            const float dopx = -kxy - k2z * k2z;
            const float dopy = dopx * dopx;
            const float inv = __frcp_rn(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
            const float2 xi = kspace_noise<float>(kx, ky, kz, nx, ny, NZ, a.seed, ctr);
            const float g = a.dt * a.namp_eff * sqrtf(-dopx) * inv;
            float2 w = scratch[kz * TX + c];
            w.x += g * xi.x;
            w.y += g * xi.y;
            scratch[kz * TX + c] = w;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) v[u * P + k2] = scratch[((t * U + u) + E * k2) * TX + c];
    }
    bool bad = false;
#pragma unroll
    for (int j = 0; j < E; ++j) bad |= !isfinite(v[j].x) || !isfinite(v[j].y);
    if (bad && valid) atomicOr(flag, 1);
}

// A' (D1 after the inverse FFT, scaled) or psi^' (D2, last step) for the thread's column
template <class Z>
__device__ __forceinline__ void store_state(float2 (&v)[Z::E], float2* A, int64_t base, int64_t zs, int t, bool valid,
                                            bool final_step) {
    constexpr int E = Z::E, P = Z::P, U = Z::U, NZ = Z::NZ;
    if (!valid) return;
    if (final_step) {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) A[base + (int64_t)((t * U + u) + E * k2) * zs] = v[u * P + k2];
    } else {
        const float s = 1.0f / (float)NZ;
#pragma unroll
        for (int j = 0; j < E; ++j) A[base + (int64_t)(t + P * j) * zs] = make_float2(v[j].x * s, v[j].y * s);
    }
}

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
    propagate<Z, BarNamed<1, TH>>(v, [&](int kz) { return regB[kz * TX + c]; }, regB, kx, ky, t, c, nx, ny, valid, a,
                                  k0, flag);
    if (!a.final_step) fft_d2_to_d1<NZ, E, TX, 1, BarNamed<1, TH>, Z::PADG>(v, t, c, regA, tw);
    store_state<Z>(v, A, base, zs, t, valid, a.final_step);
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void bar_arrive(int id, int count) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <class Z>
__global__ void __launch_bounds__(Z::T, 1) k_zpipe(float2* A, const float2* __restrict__ B, int nx, int ny, ZArgsF a,
                                                    const double2* __restrict__ k0, int* flag,
                                                    const float2* __restrict__ twg) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, U = Z::U, TH = Z::TH, T = Z::T;
    extern __shared__ __align__(16) float2 sm[];
    float2* stgA = sm;
    float2* stgB = stgA + Z::STG;
    float2* regA = stgB + Z::STG;
    float2* regB = regA + Z::REG;
    float2* nh = regB + Z::REG;
    float2* tw = nh + Z::NHS;
    const int tid = threadIdx.x;
    for (int i = tid; i < NZ; i += T) tw[i] = twg[i];
    __syncthreads();
    const int half = tid / TH;
    const int lt = tid - half * TH;
    const int c = lt % TX, t = lt / TX;
    const int nxh = nx / 2 + 1;
    const int ntx = (nxh + TX - 1) / TX;
    const int ntiles = ntx * ny;
    const int64_t zs = (int64_t)ny * nxh;
    const float2* src = half ? B : A;
    float2* stg = half ? stgB : stgA;

    // each thread stages exactly the elements it later reads: no barrier around staging
    auto issue = [&](int tile) {
        const int kxq = (tile % ntx) * TX + c;
        if (kxq < nxh) {
            const float2* g = src + (int64_t)(tile / ntx) * nxh + kxq + (int64_t)t * zs;
            float2* s = stg + t * TX + c;
#pragma unroll 1
            for (int j = 0; j < E; ++j, g += P * zs, s += P * TX) cp_async8(s, g);
        }
        cp_commit();
    };

    int tile = blockIdx.x;
    if (tile < ntiles) issue(tile);
    bool first = true;
    for (; tile < ntiles; tile += gridDim.x) {
        const int kx = (tile % ntx) * TX + c;
        const int ky = tile / ntx;
        const bool valid = kx < nxh;
        const int64_t base = (int64_t)ky * nxh + kx;
        const bool has_next = tile + (int)gridDim.x < ntiles;
        cp_wait_all();
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = valid ? stg[(t + P * j) * TX + c] : make_float2(0.f, 0.f);
        if (has_next) issue(tile + gridDim.x);  // the staging buffer is free once read
        if (half == 1) {
            fft_d1_to_d2<NZ, E, TX, -1, BarNamed<2, TH>, Z::PADG>(v, t, c, regB, tw);
            if (!first) bar_sync(4, T);  // the A half is done with the previous N^
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int k2 = 0; k2 < P; ++k2) nh[nh_slot<Z>((t * U + u) + E * k2, c)] = v[u * P + k2];
            bar_arrive(3, T);  // N^ of this tile written
        } else {
            fft_d1_to_d2<NZ, E, TX, -1, BarNamed<1, TH>, Z::PADG>(v, t, c, regA, tw);
            bar_sync(3, T);
            propagate<Z, BarNamed<1, TH>>(v, [&](int kz) { return nh[nh_slot<Z>(kz, c)]; }, regA, kx, ky, t, c, nx,
                                          ny, valid, a, k0, flag);
            if (has_next) bar_arrive(4, T);  // N^ slots free for the next tile
            if (!a.final_step) fft_d2_to_d1<NZ, E, TX, 1, BarNamed<1, TH>, Z::PADG>(v, t, c, regA, tw);
            store_state<Z>(v, A, base, zs, t, valid, a.final_step);
        }
        first = false;
    }
    cp_wait_all();
}

using Z512 = ZCfg<512, 32, 8>;
using Z256 = ZCfg<256, 16, 8>;
using Z128 = ZCfg<128, 16, 8>;
using Z64 = ZCfg<64, 8, 8>;

template <class Z>
cudaError_t zattr() {
    cudaError_t e = cudaFuncSetAttribute(k_zcol<Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::SMEM);
    if (e) return e;
    return cudaFuncSetAttribute(k_zpipe<Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::SMEM_PIPE);
}

template <class Z>
cudaError_t zlaunch(const pfc_ctx* c, void* A, const void* B, const ZPropArgs& p) {
    const double tp = 6.283185307179586232;
    ZArgsF a{(float)p.dt, (float)p.eps, (float)p.C, (float)p.namp_eff, (float)(tp / p.lx), (float)(tp / p.ly),
             (float)(tp / p.lz), p.seed, p.counter, p.dev_counter, p.use_noise, p.final_step};
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
    const int ntx = (c->nxh + Z::TX - 1) / Z::TX;
    if (c->z_pipe) {
        const int ntiles = ntx * c->ny;
        const int grid = ntiles < c->num_sms ? ntiles : c->num_sms;
        k_zpipe<Z><<<grid, Z::T, Z::SMEM_PIPE, c->stream>>>((float2*)A, (const float2*)B, c->nx, c->ny, a, c->k0,
                                                             c->flag, tw);
    } else {
        dim3 grid(ntx, c->ny);
        k_zcol<Z><<<grid, Z::T, Z::SMEM, c->stream>>>((float2*)A, (const float2*)B, c->nx, c->ny, a, c->k0, c->flag,
                                                       tw);
    }
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
