// The stepper's z pass for FP32 grids with nz in {64, 128, 192, 256, 512}: register-resident
// four-step FFTs along z on tiles of TX consecutive kx columns at one ky.
//
// Per tile: psi^ = FFT_z(A) (the carried state), N^ = FFT_z(B) (the nonlinear term),
// the semi-implicit update of eom.hpp:60-72 (stabilisation C, conserved Philox noise,
// the FP64 k = 0 mode, non-finite watchdog), then A' = IFFT_z(psi^')/nz -- or psi^'
// itself on the last step.  Half of each CTA transforms A, the other half B.
//
//  k_zcol   one tile per CTA; both halves load and transform concurrently, N^ is
//           handed over through shared memory, both halves draw the update's noise, then
//           the A half finishes alone.
#include <type_traits>
#include "bulk.cuh"
#include "pfc_ctx.h"
#include "regfft.cuh"

namespace pfc {
namespace {

struct ZArgsF {
    float dt, eps, C, namp_eff, ckx, cky, ckz;  // ck = 2 pi / L per axis
    uint64_t seed, counter;
    const unsigned long long* dev_counter;      // read instead of counter when set
    int use_noise, final_step;
    unsigned* maxc;                             // relaxations: max |psi^' - psi^| (float bits), or null
    const MemberArgs* margs;                    // batched fields: per-field eps, noise amplitude, seed
};

// The field of a batch this CTA steps (grid z): its noise counter and parameters (the
// kernels also take its k0 slot, k0 + blockIdx.z).
__device__ __forceinline__ void take_member(ZArgsF& a) {
    if (a.dev_counter) a.dev_counter += blockIdx.z;
    if (a.margs) {
        const MemberArgs m = a.margs[blockIdx.z];
        a.eps = (float)m.eps;
        a.namp_eff = (float)m.namp_eff;
        a.seed = m.seed;
    }
}

constexpr int zgcd(int a, int b) { return b == 0 ? a : zgcd(b, a % b); }

template <int NZ_, int E_, int TX_, int MINB_ = 0>
struct ZCfg {
    static constexpr int NZ = NZ_, E = E_, TX = TX_;
    static constexpr int P = NZ / E, U = E / P;
    static constexpr int TH = TX * P;  // threads per field
    static constexpr int T = 2 * TH;
    // k_zcol CTAs per SM its register cap allows: with up to 16 values per thread, 6 (128
    // threads, 85 registers) or 3 (256 threads) fit without spilling and hide the latency of
    // the update's noise; 32 values per thread keep 128 registers
    static constexpr int MINB =
        MINB_ ? MINB_ : (E > 16 ? (T <= 256 ? 2 : 1) : (T <= 128 ? 6 : (T <= 256 ? 3 : 1)));
    // exchange padding: the 32/TX t-groups of a warp hit distinct banks (U PADG = TX mod 2 TX)
    static constexpr int PADG = TX / zgcd(U, TX);
    static constexpr int REG = E * (P * TX + PADG);
    static constexpr int STG = NZ * TX;  // staging of one field tile, [z][c]
    // every kernel ends its shared memory with the twiddles W_NZ^m (NZ float2) and the
    // wavenumbers k_z of the NZ modes (NZ floats)
    static constexpr int TW = NZ;  // twiddles in the tail
    static constexpr int TAIL = TW + NZ / 2 + 4;
    static constexpr size_t SMEM = (size_t)(2 * REG + TAIL) * sizeof(float2);
    static constexpr size_t SMEM_CARRY = (size_t)(REG + STG + TAIL) * sizeof(float2);  // TH threads, one field
    // resident CTAs of k_zcarry the shared memory allows (228 KB per SM): its register cap
    static constexpr int CMINB = 4 * (SMEM_CARRY + 1024) <= 228 * 1024 ? 4 : 3;
    static_assert(TH % 32 == 0 && U * P == E && E % 2 == 0 && 32 % TX == 0, "shape");
};

// Row of mode kz in a [row][c] tile of modes (TX = 8 float2 per row: the N^ hand-over
// and the psi^ staging).  A warp touches the modes kz = t U + u + E k2 of four
// consecutive t at once; with U = 2 those rows all have the parity of u, so rows are
// swapped in pairs for odd t, which puts two t-groups in each half of the 32 banks (two
// wavefronts, the minimum for 8-byte accesses).  A permutation of the rows: no padding.
template <class Z> __device__ __forceinline__ int stg_row(int kz) {
    if constexpr (Z::U == 2) return kz ^ ((kz >> 1) & 1);
    else return kz;
}

// 1 / D(k) of the semi-implicit update (D >= 1; at most about 1e5 on the grids the z pass
// takes): the one-instruction approximate reciprocal, within 2 ulp of the quotient.
__device__ __forceinline__ float prop_inv(float d) { return __fdividef(1.0f, d); }

// Slot of mode kz in the shared table of wavenumbers: one float of padding per 128 modes,
// so that modes 128 apart (the two threads of a D3 pair) read different banks.
__device__ __forceinline__ int kz_slot(int kz) { return kz + (kz >> 7); }

// Twiddles W_NZ^m (Z::TW = NZ of them, or 2 NZ: then -W_NZ^m follow, the signed table of
// fft_d1_to_d3) and wavenumbers K(kz) = kz' 2 pi / L_z (common.hpp:27-28) of the NZ modes
// into the shared tail of a z kernel (tw, then NZ + NZ / 128 floats).
template <class Z>
__device__ __forceinline__ float* load_tail(float2* tw, const float2* __restrict__ twg, const ZArgsF& a, int tid,
                                           int nthreads) {
    constexpr int NZ = Z::NZ;
    float* kz_tab = reinterpret_cast<float*>(tw + Z::TW);
    for (int i = tid; i < NZ; i += nthreads) {
        const float2 w = twg[i];
        tw[i] = w;
        if (Z::TW == 2 * NZ) tw[NZ + i] = make_float2(-w.x, -w.y);
        kz_tab[kz_slot(i)] = (float)(i < NZ / 2 + 1 ? i : i - NZ) * a.ckz;
    }
    return kz_tab;
}

// Non-finite watchdog of a column: every output of the inverse z transform depends on
// every mode of its column, so one element per thread (all of them on the last step,
// which has no inverse transform) shows a NaN or Inf anywhere in the column.
template <class Z>
__device__ __forceinline__ void watch(const float2 (&v)[Z::E], bool all, bool valid, int* flag) {
    bool bad = !isfinite(v[0].x) || !isfinite(v[0].y);
    if (all) {
#pragma unroll
        for (int j = 1; j < Z::E; ++j) bad |= !isfinite(v[j].x) || !isfinite(v[j].y);
    }
    if (bad && valid) atomicOr(flag, 1);
}

// The update of the thread's modes kz = (t U + u) + E k2 of column kx at ky; the result
// replaces v.  kPsiInV: v holds psi^ and other(kz) returns N^; otherwise v holds N^ and
// other(kz) returns psi^.  kz_tab: K(kz) of the NZ modes (load_tail).  The noise pass
// is staged through the thread's own slots scratch[slot(kz)]; kSync puts a barrier of
// the transforming threads (bar) first, for a scratch that is an exchange buffer other
// threads may still be reading.  The k = 0 mode (register 0 of thread t = 0 in column
// kx = 0 at ky = 0, where D = 1 and the noise vanishes) is set to the FP64 value k0.
// The noise term g(k) xi(k) of the update at mode kz of column (kx, ky): the conserved
// dt namp sqrt(N) |k| / D(k), or the propagator's own gain; kxy = kx^2 + ky^2 in wavenumbers.
template <class Z, int PROP>
__device__ __forceinline__ void noise_gain_xi(int kz, int kx, int ky, float kxy, float deps, const float* kz_tab, int nx,
                                              int ny, const ZArgsF& a, uint64_t ctr, float& g, float2& xi) {
    const float k2z = kz_tab[kz_slot(kz)];
    const float dopx = -kxy - k2z * k2z;
    if constexpr (PROP == kPropConserved) {
        const float dopy = dopx * dopx;
        const float inv = prop_inv(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
        g = a.dt * a.namp_eff * sqrtf(-dopx) * inv;
    } else {
        float ca, cb, cg;
        prop_coef<PROP, float>(dopx, a.dt, deps, ca, cb, cg);
        g = a.namp_eff * cg;
    }
    xi = kspace_noise<float>(kx, ky, kz, nx, ny, Z::NZ, a.seed, ctr);
}

// noise_modes: the thread's modes m < noise_modes (mode m: kz = (t U + m / P) + E (m % P),
// register m) take their noise here; a caller that splits the noise with other threads
// adds the rest.
template <class Z, bool kPsiInV, bool kSync, int PROP, class Bar, class OTHER, class SLOT>
__device__ __forceinline__ void propagate(float2 (&v)[Z::E], OTHER other, float2* scratch, SLOT slot, const Bar& bar,
                                          const float* kz_tab, int kx, int ky, int t, int nx, int ny,
                                          const ZArgsF& a, const double2* k0, int noise_modes = Z::E) {
    constexpr int E = Z::E, P = Z::P, U = Z::U;
    // wavenumbers K(i) = i' * 2 pi / L (common.hpp:27-28) with 2 pi / L precomputed
    const float k0x = (float)kx * a.ckx;
    const float k1y = (float)(ky < ny / 2 + 1 ? ky : ky - ny) * a.cky;
    const float kxy = k0x * k0x + k1y * k1y;
    const float deps = 1.0f + a.C - a.eps;
    float mc = 0.f;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) {
            const int kz = (t * U + u) + E * k2;
            const float2 psi = kPsiInV ? v[u * P + k2] : other(kz);
            const float2 n = kPsiInV ? other(kz) : v[u * P + k2];
            const float k2z = kz_tab[kz_slot(kz)];
            const float dopx = -kxy - k2z * k2z;
            if constexpr (PROP == kPropConserved) {
                const float dopy = dopx * dopx;
                const float inv = prop_inv(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy));
                const float f = a.dt * dopx;
                v[u * P + k2] = make_float2((psi.x + f * n.x) * inv, (psi.y + f * n.y) * inv);
            } else {
                float ca, cb, cg;
                prop_coef<PROP, float>(dopx, a.dt, deps, ca, cb, cg);
                const float2 w = make_float2(ca * psi.x + cb * n.x, ca * psi.y + cb * n.y);
                if (!prop_conserved<PROP>())
                    mc = fmaxf(mc, (w.x - psi.x) * (w.x - psi.x) + (w.y - psi.y) * (w.y - psi.y));
                v[u * P + k2] = w;
            }
        }
    if (!prop_conserved<PROP>() && a.maxc) fold_max_change(sqrtf(mc), a.maxc);
    if (a.use_noise) {
        // conserved k-space noise, dt namp sqrt(N) |k| xi / D(k): a compact loop over this
        // thread's modes, staged through its own slots (kept out of the unrolled body)
        if (kSync) bar.sync();
        const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) scratch[slot((t * U + u) + E * k2)] = v[u * P + k2];
#pragma unroll 1
        for (int m = 0; m < noise_modes; ++m) {
            const int kz = (t * U + m / P) + E * (m % P);
            float g;
            float2 xi;
            noise_gain_xi<Z, PROP>(kz, kx, ky, kxy, deps, kz_tab, nx, ny, a, ctr, g, xi);
            float2 w = scratch[slot(kz)];
            w.x += g * xi.x;
            w.y += g * xi.y;
            scratch[slot(kz)] = w;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) v[u * P + k2] = scratch[slot((t * U + u) + E * k2)];
    }
    if (prop_conserved<PROP>() && kx == 0 && ky == 0 && t == 0) v[0] = make_float2((float)k0->x, (float)k0->y);
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

// lay bits 0, 1, 2: A, B, O kx-tiled (col_addr); O may be A when their layouts agree.
template <class Z, int PROP>
__global__ void __launch_bounds__(Z::T, Z::MINB) k_zcol(const float2* A, const float2* __restrict__ B, float2* O,
                                                   int nx, int ny, int lay, ZArgsF a,
                                                   const double2* __restrict__ k0, int* flag,
                                                   const float2* __restrict__ twg, int64_t ms) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, U = Z::U, TH = Z::TH;
    A += blockIdx.z * ms;  // fields of a batch (grid z)
    B += blockIdx.z * ms;
    O += blockIdx.z * ms;
    take_member(a);
    k0 += blockIdx.z;
    extern __shared__ __align__(16) float2 sm[];
    float2* regA = sm;
    float2* regB = sm + Z::REG;
    float2* tw = sm + 2 * Z::REG;
    const int tid = threadIdx.x;
    const float* kz_tab = load_tail<Z>(tw, twg, a, tid, Z::T);
    const int half = tid / TH;
    const int lt = tid - half * TH;
    const int c = lt % TX, t = lt / TX;
    const int kx = blockIdx.x * TX + c;
    const int ky = blockIdx.y;
    const int nxh = nx / 2 + 1;
    const bool valid = kx < nxh;  // the last tile holds only the kx = nx/2 column
    const float2* src = half ? B : A;
    const ColAddr ca = col_addr((lay & (half ? 2 : 1)) ? 1 : 0, true, kx, ky, nxh, ny, NZ);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? src[ca.base + (int64_t)(t + P * j) * ca.stride] : make_float2(0.f, 0.f);
    __syncthreads();
    // both halves run one copy of the forward transform, each on its own named barrier
    const BarDyn bar{1 + half, TH};
    fft_d1_to_d2<NZ, E, TX, -1, BarDyn, Z::PADG>(v, t, c, half ? regB : regA, tw, bar);
    auto own = [&](int kz) { return stg_row<Z>(kz) * TX + c; };  // N^ hand-over slots, conflict-free
    if (half != 0) {
        bar.sync();
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) regB[own((t * U + u) + E * k2)] = v[u * P + k2];
    }
    __syncthreads();
    // With noise the B half draws the noise terms g(k) xi(k) of the upper half of the column's
    // modes (m >= E/2 of the A thread with the same lt) into their slots of regA, which the A
    // half leaves idle between its two transforms; the A half draws the lower half itself and
    // adds the others after a barrier (a kernel-uniform condition: both halves take it).
    constexpr int kSplit = E / 2;
    if (half != 0) {
        if (a.use_noise) {
            const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
            const float k0x = (float)kx * a.ckx;
            const float k1y = (float)(ky < ny / 2 + 1 ? ky : ky - ny) * a.cky;
            const float kxy = k0x * k0x + k1y * k1y;
            const float deps = 1.0f + a.C - a.eps;
#pragma unroll 1
            for (int m = kSplit; m < E; ++m) {
                const int kz = (t * U + m / P) + E * (m % P);
                float g;
                float2 xi;
                noise_gain_xi<Z, PROP>(kz, kx, ky, kxy, deps, kz_tab, nx, ny, a, ctr, g, xi);
                regA[own(kz)] = make_float2(g * xi.x, g * xi.y);
            }
            __syncthreads();
        }
        return;
    }
    propagate<Z, true, true, PROP>(v, [&](int kz) { return regB[own(kz)]; }, regB, own, bar, kz_tab, kx, ky, t, nx, ny,
                                   a, k0, a.use_noise ? kSplit : E);
    if (a.use_noise) {
        __syncthreads();
#pragma unroll
        for (int m = kSplit; m < E; ++m) {
            const float2 n = regA[own((t * U + m / P) + E * (m % P))];
            v[m].x += n.x;
            v[m].y += n.y;
        }
    }
    if (!a.final_step) fft_d2_to_d1<NZ, E, TX, 1, BarDyn, Z::PADG>(v, t, c, regA, tw, bar);
    watch<Z>(v, a.final_step, valid, flag);
    const ColAddr co = col_addr((lay & 4) ? 1 : 0, true, kx, ky, nxh, ny, NZ);
    store_state<Z>(v, O, co.base, co.stride, t, valid, a.final_step);
}

// ---- the z pass with E values per thread over 2E threads per column (NZ = 2 E^2,
// fft_d1_to_d3): half the registers of k_zcol's square split, so twice the resident warps.
template <int NZ_, int E_, int TX_>
struct Z3Cfg {
    static constexpr int NZ = NZ_, E = E_, TX = TX_, P = 2 * E, TH = TX * P, T = 2 * TH;
    static constexpr int REG = E * (P + 1) * TX;  // exchange buffer of one half
    static constexpr int TW = 2 * NZ;  // the signed twiddle table of fft_d1_to_d3
    static constexpr int TAIL = TW + NZ / 2 + 4;
    static constexpr size_t SMEM = (size_t)(2 * REG + TAIL) * sizeof(float2);
    static constexpr size_t SMEM_CARRY = (size_t)(REG + NZ * TX + TAIL) * sizeof(float2);  // k_zcarry3
    static_assert(P * E == NZ && TH % 32 == 0 && REG >= NZ * TX, "shape");
};

// propagate for distribution D3: register r of thread t = 2p + h holds mode
// kz = p + h E^2/2 + d3_off(r).  kPsiInV: v holds psi^ and the tile N^, else the converse;
// the tile ([row][TX], rows as d3_off's comment, column c) is also the noise pass's scratch
// (the thread's own slots).  kSync: a barrier before that use.  sc scales the result (a
// power of two: exact), the 1/nz of a following inverse transform folded into 1/D(k).
// kPadRows: the tile holds mode kz in row kz + kz / 128 (blocks of 128 rows, each followed
// by one row of padding: the two threads of a pair, 128 modes apart, meet opposite bank
// halves) instead of the swizzled rows.
template <int E, bool kPadRows> __device__ __forceinline__ constexpr int d3_row(int r) {
    return kPadRows ? d3_off<E>(r) + (d3_off<E>(r) >> 7) : d3_off<E>(r);
}
template <class Z, bool kPsiInV, bool kSync, class Bar, bool kPadRows = false, int PROP = kPropConserved>
__device__ __forceinline__ void propagate3(float2 (&v)[Z::E], float2* tile, int c, const Bar& bar,
                                           const float* kz_tab, int kx, int ky, int t, int nx, int ny,
                                           const ZArgsF& a, const double2* k0, float sc) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, B = E * E / 2;
    static_assert(B == 128, "kz_slot pads one float per 128 modes");
    const int p = t >> 1, h = t & 1;
    const int kzb = p + h * B;                   // kz = kzb + d3_off(r)
    float2* trow = tile + (kPadRows ? p + h * (B + 1) : (p ^ h) + h * B) * TX + c;  // + d3_row(r) TX
    const float* tab = kz_tab + kzb + h;         // kz_slot(kz) = kzb + h + d3_off(r) + 2 [r >= E/2]
    const float k0x = (float)kx * a.ckx;
    const float k1y = (float)(ky < ny / 2 + 1 ? ky : ky - ny) * a.cky;
    const float kxy = k0x * k0x + k1y * k1y;
    const float deps = 1.0f + a.C - a.eps;
    float mc = 0.f;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const float2 o = trow[d3_row<E, kPadRows>(r) * TX];
        const float2 psi = kPsiInV ? v[r] : o;
        const float2 n = kPsiInV ? o : v[r];
        const float k2z = tab[d3_off<E>(r) + (r >= E / 2 ? 2 : 0)];
        const float dopx = -kxy - k2z * k2z;
        if constexpr (PROP == kPropConserved) {
            const float dopy = dopx * dopx;
            const float inv = prop_inv(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy)) * sc;
            const float f = a.dt * dopx;
            v[r] = make_float2((psi.x + f * n.x) * inv, (psi.y + f * n.y) * inv);
        } else {
            float ca, cb, cg;
            prop_coef<PROP, float>(dopx, a.dt, deps, ca, cb, cg);
            const float2 w = make_float2(ca * psi.x + cb * n.x, ca * psi.y + cb * n.y);
            if (!prop_conserved<PROP>())
                mc = fmaxf(mc, (w.x - psi.x) * (w.x - psi.x) + (w.y - psi.y) * (w.y - psi.y));
            v[r] = make_float2(w.x * sc, w.y * sc);
        }
    }
    if (!prop_conserved<PROP>() && a.maxc) fold_max_change(sqrtf(mc), a.maxc);
    if (a.use_noise) {
        if (kSync) bar.sync();
        const uint64_t ctr = a.dev_counter ? *a.dev_counter : a.counter;
#pragma unroll
        for (int r = 0; r < E; ++r) trow[d3_row<E, kPadRows>(r) * TX] = v[r];
#pragma unroll 1
        for (int r = 0; r < E; ++r) {
            const int off = r < E / 2 ? E * r : E * E + E * (r - E / 2);
            const int row = kPadRows ? off + (off >> 7) : off;
            const int kz = kzb + off;
            const float k2z = tab[off + (r >= E / 2 ? 2 : 0)];
            const float dopx = -kxy - k2z * k2z;
            float g;
            if constexpr (PROP == kPropConserved) {
                const float dopy = dopx * dopx;
                const float inv = prop_inv(1.0f - a.dt * (deps * dopx + 2.0f * dopy + dopx * dopy)) * sc;
                g = a.dt * a.namp_eff * sqrtf(-dopx) * inv;
            } else {
                float ca, cb, cg;
                prop_coef<PROP, float>(dopx, a.dt, deps, ca, cb, cg);
                g = a.namp_eff * cg * sc;
            }
            const float2 xi = kspace_noise<float>(kx, ky, kz, nx, ny, NZ, a.seed, ctr);
            float2 w = trow[row * TX];
            w.x += g * xi.x;
            w.y += g * xi.y;
            trow[row * TX] = w;
        }
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = trow[d3_row<E, kPadRows>(r) * TX];
    }
    if (prop_conserved<PROP>() && kx == 0 && ky == 0 && t == 0)
        v[0] = make_float2((float)k0->x * sc, (float)k0->y * sc);  // kz = 0 at r = 0
}

// LAY: the layouts of A, B, O as k_zcol's lay, fixed at compile time (0, 1 or 7)
template <class Z, int LAY, int PROP>
__global__ void __launch_bounds__(Z::T, 2) k_zcol3(const float2* A, const float2* __restrict__ B, float2* O, int nx,
                                                    int ny, ZArgsF a, const double2* __restrict__ k0, int* flag,
                                                    const float2* __restrict__ twg, int64_t ms) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, TH = Z::TH;
    A += blockIdx.z * ms;  // fields of a batch (grid z)
    B += blockIdx.z * ms;
    O += blockIdx.z * ms;
    take_member(a);
    k0 += blockIdx.z;
    extern __shared__ __align__(16) float2 sm[];
    float2* regA = sm;
    float2* regB = sm + Z::REG;
    float2* tw = sm + 2 * Z::REG;
    const int tid = threadIdx.x;
    const float* kz_tab = load_tail<Z>(tw, twg, a, tid, Z::T);
    const int half = tid / TH;
    const int lt = tid - half * TH;
    const int c = lt % TX, t = lt / TX;
    const int kx = blockIdx.x * TX + c;
    const int ky = blockIdx.y;
    const int nxh = nx / 2 + 1;
    const bool valid = kx < nxh;
    const float2* src = half ? B : A;
    static_assert(TX == kTileW, "the tiles of the kx-tiled layout");
    const ColAddr ca = half ? zcol_addr<(LAY & 2) != 0>(blockIdx.x, c, ky, nxh, ny, NZ)
                            : zcol_addr<(LAY & 1) != 0>(blockIdx.x, c, ky, nxh, ny, NZ);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? src[ca.base + (int64_t)(t + P * j) * ca.stride] : make_float2(0.f, 0.f);
    __syncthreads();
    const BarDyn bar{1 + half, TH};
    fft_d1_to_d3<NZ, E, TX, -1, BarDyn>(v, t, c, half ? regB : regA, tw, bar);
    const int p = t >> 1, h = t & 1;
    if (half != 0) {
        // N^ hand-over in the rows of propagate3's tile
        float2* trow = regB + ((p ^ h) + h * (E * E / 2)) * TX + c;
        bar.sync();
#pragma unroll
        for (int r = 0; r < E; ++r) trow[d3_off<E>(r) * TX] = v[r];
    }
    __syncthreads();
    if (half != 0) return;
    propagate3<Z, true, false, BarDyn, false, PROP>(v, regB, c, bar, kz_tab, kx, ky, t, nx, ny, a, k0,
                                                    a.final_step ? 1.0f : 1.0f / (float)NZ);
    if (!a.final_step) fft_d3_to_d1<NZ, E, TX, 1, BarDyn>(v, t, c, regA, tw, bar);
    watch<Z>(v, a.final_step, valid, flag);
    if (!valid) return;
    const ColAddr co = zcol_addr<(LAY & 4) != 0>(blockIdx.x, c, ky, nxh, ny, NZ);
    if (a.final_step) {
#pragma unroll
        for (int r = 0; r < E; ++r) O[co.base + (int64_t)(p + E * d3_k2<E>(r, h)) * co.stride] = v[r];
    } else {  // A' = IFFT_z(psi^')/nz, the 1/nz applied in propagate3
#pragma unroll
        for (int j = 0; j < E; ++j) O[co.base + (int64_t)(t + P * j) * co.stride] = v[j];
    }
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }


// The z pass when the state psi^ itself is carried (k-space, reference layout) and
// A = IFFT_z(psi^)/nz is only the input of the next xy part.  The whole CTA works on
// one field: psi^ of the tile is copied into a shared staging tile with cp.async while
// every thread loads and transforms B (N^ = FFT_z(B)); the update then reads psi^ from
// the staging tile (no transform), writes psi^' and, unless this is the last step,
// A' = IFFT_z(psi^')/nz.  Two z transforms per column instead of k_zcol's three, no FP32
// round trip of the state per step (its rounding matches the reference's k-space
// update), and one more read and write of the state.
template <class Z, int PROP>
__global__ void __launch_bounds__(Z::TH, Z::CMINB) k_zcarry(float2* kpsi, float2* A, const float2* __restrict__ B, int nx,
                                                      int ny, ZArgsF a, const double2* __restrict__ k0, int* flag,
                                                      const float2* __restrict__ twg, int64_t ms) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, TH = Z::TH;
    static_assert(TX == 8 && (Z::U == 1 || Z::U == 2), "staging swizzle assumes 8 columns per tile");
    kpsi += blockIdx.z * ms;  // fields of a batch (grid z)
    A += blockIdx.z * ms;
    B += blockIdx.z * ms;
    take_member(a);
    k0 += blockIdx.z;
    extern __shared__ __align__(16) float2 sm[];
    float2* xb = sm;
    float2* stg = sm + Z::REG;
    float2* tw = stg + Z::STG;
    const int tid = threadIdx.x;
    const int c = tid % TX, t = tid / TX;
    const int kx = blockIdx.x * TX + c;
    const int ky = blockIdx.y;
    const int nxh = nx / 2 + 1;
    const bool valid = kx < nxh;  // the last tile holds only the kx = nx/2 column
    const int64_t zs = (int64_t)ny * nxh;
    const int64_t base = (int64_t)ky * nxh + kx;
    if (valid) {
#pragma unroll 4
        for (int j = 0; j < E; ++j) {
            const int z = t + P * j;
            cp_async8(&stg[stg_row<Z>(z) * TX + c], kpsi + base + (int64_t)z * zs);
        }
    }
    cp_commit();
    const float* kz_tab = load_tail<Z>(tw, twg, a, tid, TH);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? B[base + (int64_t)(t + P * j) * zs] : make_float2(0.f, 0.f);
    __syncthreads();
    fft_d1_to_d2<NZ, E, TX, -1, BarCta, Z::PADG>(v, t, c, xb, tw);
    cp_wait_all();
    __syncthreads();  // psi^ staged by the other threads of the column is visible
    // the noise pass stages through the thread's own psi^ slots, read only by itself
    auto own = [&](int kz) { return stg_row<Z>(kz) * TX + c; };
    propagate<Z, false, false, PROP>(v, [&](int kz) { return stg[own(kz)]; }, stg, own, BarCta{}, kz_tab, kx, ky, t, nx,
                                     ny, a, k0);
    if (a.final_step) watch<Z>(v, true, valid, flag);
    store_state<Z>(v, kpsi, base, zs, t, valid, true);
    if (a.final_step) return;
    fft_d2_to_d1<NZ, E, TX, 1, BarCta, Z::PADG>(v, t, c, xb, tw);
    watch<Z>(v, false, valid, flag);
    store_state<Z>(v, A, base, zs, t, valid, false);
}

// The psi^-carrying z pass with 16 values per thread (fft_d1_to_d3) on the z-tiled layout,
// one field per CTA of TH threads: the psi^ block of the tile (contiguous) is staged in
// shared memory with cp.async while B is loaded and transformed; the update reads psi^
// from the stage and writes psi^' (in place), then A' = IFFT_z(psi^')/nz over B's block.
// kLast: B and psi^' in the standard layout (psi^' over B, in place), no A'.  Shared
// memory: the exchange buffer, the stage [kz][c] (a warp's four modes per register have
// two even and two odd kz: no bank conflicts), the tail.
// kt0, ky0: the kx tile and the ky of blockIdx.x = 0 and blockIdx.y = 0 (a launch may cover
// only some tiles, or some ky).
template <class Z, bool kLast, int PROP>
__global__ void __launch_bounds__(Z::TH, 3) k_zcarry3(const float2* psi_in, const float2* B, float2* psi_out,
                                                       float2* A, int nx, int ny, ZArgsF a,
                                                       const double2* __restrict__ k0, int* flag,
                                                       const float2* __restrict__ twg, int kt0, int ky0, int64_t ms) {
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, TH = Z::TH;
    static_assert(TX == kTileW, "the tiles of the z-tiled layout");
    psi_in += blockIdx.z * ms;  // fields of a batch (grid z)
    B += blockIdx.z * ms;
    psi_out += blockIdx.z * ms;
    if (A) A += blockIdx.z * ms;
    take_member(a);
    k0 += blockIdx.z;
    extern __shared__ __align__(16) float2 sm[];
    float2* xb = sm;
    float2* stg = sm + Z::REG;
    float2* tw = stg + NZ * TX;
    const int tid = threadIdx.x;
    const int c = tid % TX, t = tid / TX;
    const int kt = blockIdx.x + kt0;
    const int kx = kt * TX + c;
    const int ky = blockIdx.y + ky0;
    const int nxh = nx / 2 + 1;
    const bool valid = kx < nxh;
    const ColAddr cp = zcol_addr<true>(kt, c, ky, nxh, ny, NZ);
    const ColAddr cb = zcol_addr<!kLast>(kt, c, ky, nxh, ny, NZ);
    if (valid) {
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int z = t + P * j;
            cp_async8(&stg[((t ^ d1_flip<E>(j)) + P * j) * TX + c], psi_in + cp.base + (int64_t)z * cp.stride);
        }
    }
    cp_commit();
    const float* kz_tab = load_tail<Z>(tw, twg, a, tid, TH);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? B[cb.base + (int64_t)(t + P * j) * cb.stride] : make_float2(0.f, 0.f);
    __syncthreads();
    fft_d1_to_d3<NZ, E, TX, -1>(v, t, c, xb, tw);
    cp_wait_all();
    __syncthreads();  // psi^ staged by the other threads of the column is visible
    propagate3<Z, false, false, BarCta, false, PROP>(v, stg, c, BarCta{}, kz_tab, kx, ky, t, nx, ny, a, k0, 1.0f);
    const int p = t >> 1, h = t & 1;
    if (kLast) watch<Z>(v, true, valid, flag);
    if (valid) {
        const ColAddr co = kLast ? cb : cp;
#pragma unroll
        for (int r = 0; r < E; ++r) psi_out[co.base + (int64_t)(p + E * d3_k2<E>(r, h)) * co.stride] = v[r];
    }
    if (kLast) return;
    fft_d3_to_d1<NZ, E, TX, 1>(v, t, c, xb, tw);
    watch<Z>(v, false, valid, flag);
    if (valid) {
        const float s = 1.0f / (float)NZ;
#pragma unroll
        for (int j = 0; j < E; ++j) A[cb.base + (int64_t)(t + P * j) * cb.stride] = make_float2(v[j].x * s, v[j].y * s);
    }
}

// The psi^-carrying z pass on whole kx tiles of the z-tiled layout with bulk asynchronous
// copies (the TMA unit) for every byte it moves: per CTA (one tile of TX = 8 columns at one
// ky, 32 threads per column, 16 values per thread) the psi^ block and the B block, each
// one contiguous 32 KB block, arrive in shared memory on one mbarrier while the CTA loads
// its twiddles; N^ = FFT_z(B) in registers; the update reads psi^ from shared memory and
// writes psi^' back in place, which one bulk copy per 128 modes stores; A' = IFFT_z(psi^')
// / nz goes through shared memory into one bulk store over B's block.  No thread issues a
// global load or store of field data.  Shared memory (float2 units): psi^ in four pieces
// of 128 kz rows of TX, each followed by a row of padding (kz at row kz + kz / 128); the B
// stage, reused as the unpadded exchange buffer and as the A' stage; the signed twiddles;
// the wavenumbers; the mbarrier.  About 75 KB: three CTAs per SM.
template <class Z>
struct ZBulkCfg {
    static constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, TH = Z::TH;
    static constexpr int PIECE = 128;                        // kz rows per bulk piece of psi^
    static constexpr int NPIECE = NZ / PIECE;
    static constexpr int STP = NPIECE * (PIECE + 1) * TX;    // psi^ stage
    static constexpr int XB = E * P * TX;                    // B stage / exchange (PADX = 0)
    static constexpr int TAIL = Z::TW + NZ / 2 + 2;          // twiddles, NZ + NZ/128 floats
    static constexpr size_t SMEM = (size_t)(STP + XB + TAIL) * sizeof(float2) + 16;
    static_assert(XB == NZ * TX && NZ % PIECE == 0 && TX == kTileW, "shape");
};

template <class Z, int PROP>
__global__ void __launch_bounds__(Z::TH, 3) k_zbulk(float2* psi, float2* BA, int nx, int ny, ZArgsF a,
                                                     const double2* __restrict__ k0, int* flag,
                                                     const float2* __restrict__ twg, int64_t ms) {
    psi += blockIdx.z * ms;  // fields of a batch (grid z)
    BA += blockIdx.z * ms;
    take_member(a);
    k0 += blockIdx.z;
    using C = ZBulkCfg<Z>;
    constexpr int NZ = Z::NZ, E = Z::E, TX = Z::TX, P = Z::P, TH = Z::TH;
    extern __shared__ __align__(16) float2 sm[];
    float2* stp = sm;
    float2* xb = sm + C::STP;
    float2* tw = xb + C::XB;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + C::TAIL);
    const int tid = threadIdx.x;
    const int c = tid % TX, t = tid / TX;
    const int kt = blockIdx.x, ky = blockIdx.y;
    const int kx = kt * TX + c;
    const int nxh = nx / 2 + 1;
    // the tile's blocks: [z][c] rows of TX (a whole tile: wt = TX)
    const int64_t blk = ((int64_t)kt * TX * ny + (int64_t)ky * TX) * NZ;
    constexpr unsigned kBlockBytes = NZ * TX * sizeof(float2);
    constexpr unsigned kPieceBytes = C::PIECE * TX * sizeof(float2);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
        mbar_arrive_expect_tx(bar, 2 * kBlockBytes);
#pragma unroll
        for (int q = 0; q < C::NPIECE; ++q)
            bulk_load(stp + q * (C::PIECE + 1) * TX, psi + blk + q * C::PIECE * TX, kPieceBytes, bar);
        bulk_load(xb, BA + blk, kBlockBytes, bar);
    }
    const float* kz_tab = load_tail<Z>(tw, twg, a, tid, TH);
    __syncthreads();  // the tail, and the barrier's initialisation
    if (!mbar_wait(bar, 0, kWaitPolls)) {
        if (tid == 0) atomicOr(flag, kFlagWaitTimeout);
        return;
    }
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = xb[(t + P * j) * TX + c];
    // (fft_d1_to_d3 synchronises before its first write to xb)
    fft_d1_to_d3<NZ, E, TX, -1, BarCta, true, 0>(v, t, c, xb, tw);
    propagate3<Z, false, false, BarCta, true, PROP>(v, stp, c, BarCta{}, kz_tab, kx, ky, t, nx, ny, a, k0, 1.0f);
    {
        // psi^' over psi^ in the thread's own slots (the rows it read), then to the async proxy
        const int p = t >> 1, h = t & 1;
        float2* trow = stp + (p + h * (C::PIECE + 1)) * TX + c;
#pragma unroll
        for (int r = 0; r < E; ++r) trow[d3_row<E, true>(r) * TX] = v[r];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < C::NPIECE; ++q)
            bulk_store(psi + blk + q * C::PIECE * TX, stp + q * (C::PIECE + 1) * TX, kPieceBytes);
        bulk_commit();
    }
    fft_d3_to_d1<NZ, E, TX, 1, BarCta, 0>(v, t, c, xb, tw);
    watch<Z>(v, false, kx < nxh, flag);
    const float s = 1.0f / (float)NZ;
    __syncthreads();  // every thread's last exchange reads are done
#pragma unroll
    for (int j = 0; j < E; ++j) xb[(t + P * j) * TX + c] = make_float2(v[j].x * s, v[j].y * s);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        bulk_store(BA + blk, xb, kBlockBytes);
        bulk_commit();
        bulk_wait_read();  // shared memory stays valid until both stores have read it
    }
}

// Copy between the standard and the z-tiled layouts (col_addr layouts 0, 1): one kx tile
// of the z columns at one ky per CTA of TX * 32 threads.
__global__ void __launch_bounds__(256) k_relayout(const float2* __restrict__ in, float2* __restrict__ out, int nxh,
                                                  int ny, int nz, int to_tiled, int ky0) {
    const int c = threadIdx.x % kTileW, t = threadIdx.x / kTileW;
    const int kt = blockIdx.x, ky = blockIdx.y + ky0;
    if (kt * kTileW + c >= nxh) return;
    const ColAddr s = to_tiled ? zcol_addr<false>(kt, c, ky, nxh, ny, nz) : zcol_addr<true>(kt, c, ky, nxh, ny, nz);
    const ColAddr d = to_tiled ? zcol_addr<true>(kt, c, ky, nxh, ny, nz) : zcol_addr<false>(kt, c, ky, nxh, ny, nz);
    for (int z = t; z < nz; z += 32) out[d.base + (int64_t)z * d.stride] = in[s.base + (int64_t)z * s.stride];
}

using Z512 = ZCfg<512, 32, 8>;
using Z3_512 = Z3Cfg<512, 16, 8>;  // 16 values per thread (k_zcol3)
using Z256 = ZCfg<256, 16, 8>;
using Z128 = ZCfg<128, 16, 8>;
using Z64 = ZCfg<64, 8, 8>;
using Z192 = ZCfg<192, 24, 8, 6>;  // P 8, U 3 (the first stage a radix-3 step); 80 registers

// The propagator of a launch as a compile-time constant: f(std::integral_constant<int, PROP>).
template <class F>
cudaError_t by_prop(int prop, F&& f) {
    switch (prop) {
        case kPropConservedExp: return f(std::integral_constant<int, kPropConservedExp>{});
        case kPropRelax: return f(std::integral_constant<int, kPropRelax>{});
        case kPropRelaxExp: return f(std::integral_constant<int, kPropRelaxExp>{});
        case kPropConservedPoly: return f(std::integral_constant<int, kPropConservedPoly>{});
        default: return f(std::integral_constant<int, kPropConserved>{});
    }
}
// f(k) for the kernel of every propagator (attribute set-up)
template <class F>
cudaError_t each_prop(F&& f) {
    cudaError_t e = cudaSuccess;
    for (int p = 0; p <= kPropConservedPoly && !e; ++p) e = by_prop(p, f);
    return e;
}

template <class Z>
cudaError_t zattr() {
    return each_prop([](auto P) {
        cudaError_t e = cudaFuncSetAttribute(k_zcol<Z, P.value>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)Z::SMEM);
        if constexpr (Z::U == 1 || Z::U == 2) {  // (k_zcarry: U of 1 or 2 only)
            if (e) return e;
            return cudaFuncSetAttribute(k_zcarry<Z, P.value>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)Z::SMEM_CARRY);
        }
        return e;
    });
}

ZArgsF zargs_f(const ZPropArgs& p) {
    const double tp = 6.283185307179586232;
    return ZArgsF{(float)p.dt, (float)p.eps, (float)p.C, (float)p.namp_eff, (float)(tp / p.lx), (float)(tp / p.ly),
                  (float)(tp / p.lz), p.seed, p.counter, p.dev_counter, p.use_noise, p.final_step, p.maxc, p.margs};
}

template <class Z>
cudaError_t zlaunch_carry(const pfc_ctx* c, void* kpsi, void* A, const void* B, const ZPropArgs& p) {
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
    dim3 grid((c->nxh + Z::TX - 1) / Z::TX, c->ny, c->batch);
    return by_prop(p.prop, [&](auto P) {
        k_zcarry<Z, P.value><<<grid, Z::TH, Z::SMEM_CARRY, c->stream>>>(
            (float2*)kpsi, (float2*)A, (const float2*)B, c->nx, c->ny, zargs_f(p), c->k0, c->flag, tw, c->mstride);
        return cudaGetLastError();
    });
}

template <class Z>
cudaError_t zlaunch(const pfc_ctx* c, const void* A, const void* B, void* O, const ZPropArgs& p, int lay) {
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
    dim3 grid((c->nxh + Z::TX - 1) / Z::TX, c->ny, c->batch);
    return by_prop(p.prop, [&](auto P) {
        k_zcol<Z, P.value><<<grid, Z::T, Z::SMEM, c->stream>>>((const float2*)A, (const float2*)B, (float2*)O, c->nx,
                                                                c->ny, lay, zargs_f(p), c->k0, c->flag, tw,
                                                                c->mstride);
        return cudaGetLastError();
    });
}

}  // namespace

// Register z kernels by length: 6 (nz = 512) 16 values per thread over 32 threads per
// column (fft_d1_to_d3); 1-4 the square split for 512 (psi^-carrying, standard layout
// only), 256, 128, 64.
// whether the register z pass of variant v has the psi^-carrying form in the reference
// layout (k_zcarry: U of 1 or 2)
bool zcarry_available(int v) { return v >= 1 && v <= 4; }

int fused_z_variant(int nx, int nz, int dtype) {
    if (dtype != PFC_F32 || nx < 16 || (nx / 2) % 8 != 0 || nx % 2 != 0) return 0;
    // (nz = 96: 4 threads per column leave too few warps for the update's noise; the
    // general z pass is faster there)
    switch (nz) {
        case 512: return 6;
        case 256: return 2;
        case 128: return 3;
        case 64: return 4;
        case 192: return 10;
    }
    return 0;
}

cudaError_t set_zcol_attributes(const pfc_ctx* c) {
    switch (c->fused_z) {
        case 1: return zattr<Z512>();
        case 2: return zattr<Z256>();
        case 3: return zattr<Z128>();
        case 4: return zattr<Z64>();
        case 10: return zattr<Z192>();
        case 6:
            return each_prop([](auto P) {
                using Z = Z3_512;
                const int sm = (int)Z::SMEM, smc = (int)Z::SMEM_CARRY, smb = (int)ZBulkCfg<Z>::SMEM;
                const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
                cudaError_t e = cudaFuncSetAttribute(k_zcol3<Z, 0, P.value>, attr, sm);
                if (!e) e = cudaFuncSetAttribute(k_zcol3<Z, 1, P.value>, attr, sm);
                if (!e) e = cudaFuncSetAttribute(k_zcol3<Z, 7, P.value>, attr, sm);
                if (!e) e = cudaFuncSetAttribute(k_zcarry3<Z, false, P.value>, attr, smc);
                if (!e) e = cudaFuncSetAttribute(k_zcarry3<Z, true, P.value>, attr, smc);
                if (!e) e = cudaFuncSetAttribute(k_zbulk<Z, P.value>, attr, smb);
                return e;
            });
    }
    return cudaSuccess;
}

cudaError_t launch_zcarry(const pfc_ctx* c, void* kpsi, void* A, const void* B, const ZPropArgs& a) {
    switch (c->fused_z) {
        case 1: return zlaunch_carry<Z512>(c, kpsi, A, B, a);
        case 2: return zlaunch_carry<Z256>(c, kpsi, A, B, a);
        case 3: return zlaunch_carry<Z128>(c, kpsi, A, B, a);
        case 4: return zlaunch_carry<Z64>(c, kpsi, A, B, a);
    }
    return cudaErrorNotSupported;
}

cudaError_t launch_zcarry_tiled(const pfc_ctx* c, const void* psi_in, const void* B, void* psi_out, void* A,
                                const ZPropArgs& a) {
    if (c->fused_z != 6) return cudaErrorNotSupported;
    using Z = Z3_512;
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
    const ZArgsF za = zargs_f(a);
    const int ntx = (c->nxh + Z::TX - 1) / Z::TX;
    return by_prop(a.prop, [&](auto P) {
        if (a.final_step) {
            k_zcarry3<Z, true, P.value><<<dim3(ntx, c->ny, c->batch), Z::TH, Z::SMEM_CARRY, c->stream>>>(
                (const float2*)psi_in, (const float2*)B, (float2*)psi_out, (float2*)A, c->nx, c->ny, za, c->k0,
                c->flag, tw, 0, 0, c->mstride);
            return cudaGetLastError();
        }
        // whole tiles with bulk copies (psi^ in place, A' over B); the partial last tile with
        // per-thread accesses, on the side stream beside them (the two write disjoint tiles)
        const int full = c->nxh / Z::TX;
        if (psi_in != psi_out || B != A) return cudaErrorNotSupported;
        const bool side = full > 0 && full < ntx && c->side_stream;
        cudaError_t e = cudaSuccess;
        if (side) {
            if ((e = cudaEventRecord(c->side_fork, c->stream))) return e;
            if ((e = cudaStreamWaitEvent(c->side_stream, c->side_fork, 0))) return e;
        }
        if (full < ntx)
            k_zcarry3<Z, false, P.value>
                <<<dim3(ntx - full, c->ny, c->batch), Z::TH, Z::SMEM_CARRY, side ? c->side_stream : c->stream>>>(
                    (const float2*)psi_in, (const float2*)B, (float2*)psi_out, (float2*)A, c->nx, c->ny, za, c->k0,
                    c->flag, tw, full, 0, c->mstride);
        if ((e = cudaGetLastError())) return e;
        if (full > 0)
            k_zbulk<Z, P.value><<<dim3(full, c->ny, c->batch), Z::TH, ZBulkCfg<Z>::SMEM, c->stream>>>(
                (float2*)psi_out, (float2*)A, c->nx, c->ny, za, c->k0, c->flag, tw, c->mstride);
        if ((e = cudaGetLastError())) return e;
        if (side) {
            if ((e = cudaEventRecord(c->side_join, c->side_stream))) return e;
            if ((e = cudaStreamWaitEvent(c->stream, c->side_join, 0))) return e;
        }
        return cudaSuccess;
    });
}

cudaError_t launch_relayout(const pfc_ctx* c, const void* in, void* out, int to_tiled, int ky0, int nky) {
    if (c->dtype != PFC_F32 || in == out) return cudaErrorNotSupported;
    if (nky < 0) nky = c->ny - ky0;
    if (ky0 < 0 || nky < 1 || ky0 + nky > c->ny) return cudaErrorInvalidValue;
    dim3 grid((c->nxh + kTileW - 1) / kTileW, nky);
    k_relayout<<<grid, 256, 0, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->ny, c->nz, to_tiled, ky0);
    return cudaGetLastError();
}

cudaError_t launch_zcol(const pfc_ctx* c, const void* A, const void* B, void* O, const ZPropArgs& a, int lay) {
    switch (c->fused_z) {
        case 6: {
            using Z = Z3_512;
            const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->zcol_tw_off;
            dim3 grid((c->nxh + Z::TX - 1) / Z::TX, c->ny, c->batch);
            if (lay != 0 && lay != 1 && lay != 7) return cudaErrorNotSupported;
            return by_prop(a.prop, [&](auto P) {
                auto k = lay == 7 ? k_zcol3<Z, 7, P.value> : lay == 1 ? k_zcol3<Z, 1, P.value> : k_zcol3<Z, 0, P.value>;
                k<<<grid, Z::T, Z::SMEM, c->stream>>>((const float2*)A, (const float2*)B, (float2*)O, c->nx, c->ny,
                                                      zargs_f(a), c->k0, c->flag, tw, c->mstride);
                return cudaGetLastError();
            });
        }
        case 1: return zlaunch<Z512>(c, A, B, O, a, lay);
        case 2: return zlaunch<Z256>(c, A, B, O, a, lay);
        case 3: return zlaunch<Z128>(c, A, B, O, a, lay);
        case 4: return zlaunch<Z64>(c, A, B, O, a, lay);
        case 10: return zlaunch<Z192>(c, A, B, O, a, lay);
    }
    return cudaErrorNotSupported;
}

}  // namespace pfc
