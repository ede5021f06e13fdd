// Register-resident FFT building blocks of the fused plane and column kernels.
//
//  RF<N, DIR>::run(v)     N-point DFT (N = 2^a 3^b 5^c, at most 64) of v[0..N) held in
//                         registers, natural order in and out: a radix-3 or radix-5
//                         step first where N has the factor, then radix-4 decimation in
//                         time down to 8/4/2-point kernels; every twiddle is a
//                         compile-time constant (trivial ones cost nothing).
//  fft_d1_to_d2 / fft_d2_to_d1
//                         an N-point FFT spread over P = N/E threads holding E values
//                         each (the four-step algorithm: E-point DFTs in registers,
//                         twiddles W_N^{ab}, one transpose through shared memory,
//                         P-point DFTs).  Distribution D1: thread t holds x[t + P j];
//                         distribution D2: thread t holds x[(t E/P + u) + E k2] at
//                         register u P + k2.  d1_to_d2 maps D1 input to D2 output,
//                         d2_to_d1 the converse, so an inverse FFT, a pointwise map and
//                         a forward FFT chain with no extra exchange.
#pragma once
#include <type_traits>
#include "pfc_internal.cuh"

namespace pfc {
namespace ct {
constexpr double kPi = 3.14159265358979323846264338327950288;
// Taylor series on |r| <= pi/4 (error < 1e-19), after reduction by quadrant.
constexpr double sin_s(double x) {
    double t = x, s = x;
    for (int n = 1; n < 14; ++n) { t *= -x * x / ((2.0 * n) * (2.0 * n + 1.0)); s += t; }
    return s;
}
constexpr double cos_s(double x) {
    double t = 1.0, s = 1.0;
    for (int n = 1; n < 14; ++n) { t *= -x * x / ((2.0 * n - 1.0) * (2.0 * n)); s += t; }
    return s;
}
constexpr double cos2pi(long k, long n) {
    k %= n;
    if (k < 0) k += n;
    const long q = (8 * k + n) / (2 * n);
    const double r = 2.0 * kPi * ((double)(4 * k - q * n) / (double)(4 * n));
    const double c = cos_s(r), s = sin_s(r);
    switch (q & 3) { case 0: return c; case 1: return -s; case 2: return -c; default: return s; }
}
constexpr double sin2pi(long k, long n) {
    k %= n;
    if (k < 0) k += n;
    const long q = (8 * k + n) / (2 * n);
    const double r = 2.0 * kPi * ((double)(4 * k - q * n) / (double)(4 * n));
    const double c = cos_s(r), s = sin_s(r);
    switch (q & 3) { case 0: return s; case 1: return c; case 2: return -s; default: return -c; }
}
}  // namespace ct

template <int N, int K, int DIR> struct Tw {  // exp(DIR 2 pi i K / N)
    static constexpr float re = (float)ct::cos2pi(K, N);
    static constexpr float im = (float)(DIR * ct::sin2pi(K, N));
};

template <int I, int N, class F> __device__ __forceinline__ void sfor(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        sfor<I + 1, N>(f);
    }
}

// a * exp(DIR 2 pi i K / N) with the trivial angles special-cased at compile time
template <int N, int K, int DIR> __device__ __forceinline__ float2 twmul(float2 a) {
    constexpr int k = ((K % N) + N) % N;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (4 * k == N) {
        return rot<DIR>(a);
    } else if constexpr (2 * k == N) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * k == 3 * N) {
        return rot<-DIR>(a);
    } else {
        constexpr float c = Tw<N, k, DIR>::re, s = Tw<N, k, DIR>::im;
        return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

template <int N, int DIR> struct RF;
template <int DIR> struct RF<1, DIR> { __device__ __forceinline__ static void run(float2*) {} };
template <int DIR> struct RF<2, DIR> { __device__ __forceinline__ static void run(float2* v) { Dft<float, DIR, 2>::run(v); } };
template <int DIR> struct RF<4, DIR> { __device__ __forceinline__ static void run(float2* v) { Dft<float, DIR, 4>::run(v); } };
template <int DIR> struct RF<8, DIR> { __device__ __forceinline__ static void run(float2* v) { Dft<float, DIR, 8>::run(v); } };
// Powers of two from 16 up: radix-4 steps down to the hand-written 8, 4, 2.
template <int N, int DIR> struct RF4 {
    static_assert(N % 4 == 0 && N >= 16, "power of two");
    __device__ __forceinline__ static void run(float2* v) {
        constexpr int Q = N / 4;
        float2 s0[Q], s1[Q], s2[Q], s3[Q];
#pragma unroll
        for (int m = 0; m < Q; ++m) { s0[m] = v[4 * m]; s1[m] = v[4 * m + 1]; s2[m] = v[4 * m + 2]; s3[m] = v[4 * m + 3]; }
        RF<Q, DIR>::run(s0);
        RF<Q, DIR>::run(s1);
        RF<Q, DIR>::run(s2);
        RF<Q, DIR>::run(s3);
        sfor<0, Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            const float2 a0 = s0[k];
            const float2 a1 = twmul<N, k, DIR>(s1[k]);
            const float2 a2 = twmul<N, 2 * k, DIR>(s2[k]);
            const float2 a3 = twmul<N, 3 * k, DIR>(s3[k]);
            const float2 t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = rot<DIR>(a1 - a3);
            v[k] = t0 + t2;
            v[k + 2 * Q] = t0 - t2;
            v[k + Q] = t1 + t3;
            v[k + 3 * Q] = t1 - t3;
        });
    }
};

// N = R Q with a radix R of 3 or 5 first (decimation in time): the R sub-sequences
// v[R m + r] transformed (length Q), twiddled by W_N^(r k), and combined by R-point DFTs
// into v[k + q Q].
template <int N, int DIR, int R> struct RFR {
    __device__ __forceinline__ static void run(float2* v);
};
// Lengths 2^a 3^b 5^c: powers of two by RF4, others by one radix-3 or radix-5 step first.
template <int N, int DIR> struct RF {
    __device__ __forceinline__ static void run(float2* v) {
        if constexpr ((N & (N - 1)) == 0) {
            RF4<N, DIR>::run(v);
        } else if constexpr (N % 3 == 0) {
            RFR<N, DIR, 3>::run(v);
        } else {
            static_assert(N % 5 == 0, "lengths 2^a 3^b 5^c");
            RFR<N, DIR, 5>::run(v);
        }
    }
};
template <int N, int DIR, int R>
__device__ __forceinline__ void RFR<N, DIR, R>::run(float2* v) {
    constexpr int Q = N / R;
    float2 s[R][Q];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int m = 0; m < Q; ++m) s[r][m] = v[R * m + r];
#pragma unroll
    for (int r = 0; r < R; ++r) RF<Q, DIR>::run(s[r]);
    sfor<0, Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        float2 a[R];
        sfor<0, R>([&](auto rr) {
            constexpr int r = decltype(rr)::value;
            a[r] = twmul<N, r * k, DIR>(s[r][k]);
        });
        Dft<float, DIR, R>::run(a);
#pragma unroll
        for (int q = 0; q < R; ++q) v[k + q * Q] = a[q];
    });
}

// Barrier policies of the exchanges: the whole CTA, or a named barrier over the
// first COUNT threads (used when half of a CTA runs a transform alone).
struct BarCta {
    __device__ __forceinline__ static void sync() { __syncthreads(); }
};
template <int ID, int COUNT> struct BarNamed {
    __device__ __forceinline__ static void sync() { asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(COUNT) : "memory"); }
};
// A named barrier whose id is chosen at run time: the thread groups of a CTA that run the
// same transform on different data share one copy of its code.
struct BarDyn {
    int id, count;
    __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }
};

// Distributed shared memory: the 32-bit shared::cluster address of `local` in CTA
// `rank` of this cluster, and an 8-byte store to it.
__device__ __forceinline__ uint32_t dsmem_addr(const void* local, uint32_t rank) {
    uint32_t a = (uint32_t)__cvta_generic_to_shared(local), r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void dsmem_st(uint32_t addr, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}

// L2 prefetch of the bytes [p, p + n), widened to 16-byte bounds: the buffer holding
// them must start on a 16-byte boundary and span a multiple of 16 bytes, so that the
// widened range stays inside it.  A hint: nothing waits on it.
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned n) {
    const uintptr_t a = (uintptr_t)p & ~(uintptr_t)15;
    const uintptr_t e = ((uintptr_t)p + n + 15) & ~(uintptr_t)15;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// Layouts of a half-spectrum field of nxh x ny x nz complex modes (nxh = nx/2 + 1):
//  0 standard    [z][ky][kx], cuFFT's R2C output;
//  1 z-tiled     tiles of kTileW consecutive kx; tile kt stores [ky][z][c], c < wt =
//                min(kTileW, nxh - kTileW kt), the tiles in kx order.  A z column segment of
//                a tile (all z at one ky) is one contiguous block of nz wt elements: the
//                stepper's z pass reads and writes whole blocks instead of 64-byte pieces
//                one plane (about 1 MB) apart;
//  2 row-tiled   the same tiles storing [z][y][c]: the y column segment of a tile (all y
//                at one z) is one contiguous block, and R consecutive x rows are one block
//                of R wt elements per tile.
// All three hold the same nxh ny nz elements.  col_addr: element s of the column of mode
// kx at q (q = ky for z columns, q = z for y columns) sits at base + s * stride.
constexpr int kTileW = 8;
struct ColAddr {
    int64_t base, stride;
};
__device__ __forceinline__ ColAddr col_addr(int layout, bool zaxis, int kx, int q, int nxh, int ny, int nz) {
    if (layout == 0)
        return zaxis ? ColAddr{(int64_t)q * nxh + kx, (int64_t)ny * nxh}
                     : ColAddr{(int64_t)q * ny * nxh + kx, (int64_t)nxh};
    const int kt = kx / kTileW, c = kx - kt * kTileW;
    const int wt = min(kTileW, nxh - kt * kTileW);
    const int64_t tb = (int64_t)kt * kTileW * ny * nz + c;
    if (layout == 1)
        return zaxis ? ColAddr{tb + (int64_t)q * nz * wt, (int64_t)wt}
                     : ColAddr{tb + (int64_t)q * wt, (int64_t)nz * wt};
    return zaxis ? ColAddr{tb + (int64_t)q * wt, (int64_t)ny * wt} : ColAddr{tb + (int64_t)q * ny * wt, (int64_t)wt};
}
// The z column of column c of kx tile kt at ky, for kernels whose tiles are the layout's
// (kt uniform over the CTA): the same address as col_addr with fewer live values.
template <bool kTiled>
__device__ __forceinline__ ColAddr zcol_addr(int kt, int c, int ky, int nxh, int ny, int nz) {
    if (!kTiled) return ColAddr{(int64_t)ky * nxh + kt * kTileW + c, (int64_t)ny * nxh};
    const int wt = min(kTileW, nxh - kt * kTileW);
    return ColAddr{((int64_t)kt * kTileW * ny + ky * wt) * nz + c, (int64_t)wt};
}

// Exchange slots: group g of NG interleaved groups, logical index (a, b) of an
// E x P matrix -> (a P + b) NG + a PADG + g.  Warps run over consecutive g (and, when
// NG < 32, over 32/NG consecutive t); PADG shifts successive blocks of P rows so that
// the t-groups of a warp land in different banks.  Buffer: E (P NG + PADG) float2.
template <int N, int E, int NG, int PADG>
__device__ __forceinline__ int xslot(int a, int b, int g) {
    return (a * (N / E) + b) * NG + a * PADG + g;
}

template <int N, int E, int NG, int DIR, class Bar = BarCta, int PADG = 0>
__device__ __forceinline__ void fft_d1_to_d2(float2 (&v)[E], int t, int g, float2* xb, const float2* twN,
                                             const Bar& bar = Bar{}) {
    constexpr int P = N / E, U = E / P;
    static_assert(P * E == N && U * P == E, "four-step shape");
    RF<E, DIR>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) {
        float2 w = twN[t * k1];  // t k1 < N: no wrap, a running index
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    bar.sync();
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) xb[xslot<N, E, NG, PADG>(k1, t, g)] = v[k1];
    bar.sync();
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int tt = 0; tt < P; ++tt) v[u * P + tt] = xb[xslot<N, E, NG, PADG>(t * U + u, tt, g)];
#pragma unroll
    for (int u = 0; u < U; ++u) RF<P, DIR>::run(&v[u * P]);
}

template <int N, int E, int NG, int DIR, class Bar = BarCta, int PADG = 0>
__device__ __forceinline__ void fft_d2_to_d1(float2 (&v)[E], int t, int g, float2* xb, const float2* twN,
                                             const Bar& bar = Bar{}) {
    constexpr int P = N / E, U = E / P;
    static_assert(P * E == N && U * P == E, "four-step shape");
#pragma unroll
    for (int u = 0; u < U; ++u) RF<P, DIR>::run(&v[u * P]);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int n1 = t * U + u;
#pragma unroll
        for (int k2 = 1; k2 < P; ++k2) {
            float2 w = twN[n1 * k2];  // n1 k2 < E P = N
            if (DIR > 0) w.y = -w.y;
            v[u * P + k2] = cmul(v[u * P + k2], w);
        }
    }
    bar.sync();
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) xb[xslot<N, E, NG, PADG>(t * U + u, k2, g)] = v[u * P + k2];
    bar.sync();
#pragma unroll
    for (int n1 = 0; n1 < E; ++n1) v[n1] = xb[xslot<N, E, NG, PADG>(n1, t, g)];
    RF<E, DIR>::run(v);
}

// ---- N = E x 2E over P = 2E threads holding E values each (half the registers of the
// square four-step above, for N = 2 E^2: 512 = 16 x 32, 128 = 8 x 16).
// Stage 1: E-point DFTs in registers, twiddles W_N^{t k1}, a transpose through shared
// memory.  Stage 2: the 2E-point DFTs over t (one per k1) split across thread pairs
// s = 2p + h (p = k1): thread h takes the E-point DFT of the t = 2m + h inputs, and the
// radix-2 combination with W_2E^{k2} exchanges half of the values with the partner through
// one round of warp shuffles (the partner is NG lanes away).
// D1: thread t holds x[t + P j].  D3: thread (p, h) holds X[p + E k2] with
// k2 = h E/2 + i at register i and k2 = E + h E/2 + i at register E/2 + i (i < E/2).
// Balance of the radix-2 step: the t = 2m + 1 values reach thread h = 1 multiplied by
// (-1)^m, which rotates its E-point DFT by E/2 (F[(k + E/2) mod E] at register k, since
// (-1)^m = W_E^{m E/2}).  Both threads of a pair then send register E/2 + i, and each
// applies E/2 of the W_2E twiddles.  The inverse keeps thread h = 1's B values rotated the
// same way, so its outputs carry (-1)^m, removed by their readers.  Each sign rides on the
// stage-1 twiddles: twN holds W_N^m for m < N, then -W_N^m, and a thread of odd t with odd
// t/2 takes its twiddles from the second half (k1 = 0 included: twN[N] = -1).
// Exchange slots (k1, t, g) -> (k1 P + t) NG + k1 NG PADX + g: with PADX = 1 a pad of NG
// per k1 row puts the four (p, h) of a warp in alternate halves of the banks.  Buffer:
// E (P + PADX) NG.
template <int N, int E, int NG, int PADX = 1>
__device__ __forceinline__ int xslot3(int k1, int t, int g) {
    return (k1 * (2 * E) + t) * NG + k1 * NG * PADX + g;
}

// the stage-1 twiddles of D1 thread t (signed as above)
template <int N> __device__ __forceinline__ const float2* d3_tw1(const float2* twN, int t) {
    return twN + ((t & 1) & ((t >> 1) & 1)) * N;
}

// kBal false: the same transform without the balance (twN of N entries; thread h = 1 applies
// all E - 1 W_2E twiddles and the pair selects what it sends).
template <int N, int E, int NG, int DIR, class Bar = BarCta, bool kBal = true, int PADX = 1>
__device__ __forceinline__ void fft_d1_to_d3(float2 (&v)[E], int t, int g, float2* xb, const float2* twN,
                                             const Bar& bar = Bar{}) {
    constexpr int P = 2 * E, H = E / 2;
    static_assert(P * E == N && (E & (E - 1)) == 0 && NG <= 16 && 32 % NG == 0, "shape");
    RF<E, DIR>::run(v);
    const float2* tw1 = kBal ? d3_tw1<N>(twN, t) : twN;
    if (kBal) {
        const float s0 = tw1[0].x;  // +-1
        v[0] = make_float2(v[0].x * s0, v[0].y * s0);
    }
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) {
        float2 w = tw1[t * k1];  // t k1 < N: no wrap, a running index
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    bar.sync();
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) xb[xslot3<N, E, NG, PADX>(k1, t, g)] = v[k1];
    bar.sync();
    const int p = t >> 1, h = t & 1;
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = xb[xslot3<N, E, NG, PADX>(p, 2 * m + h, g)];
    RF<E, DIR>::run(v);  // h = 0: F0[k] at k; h = 1: F1[(k + H) mod E] at k (kBal)
    if constexpr (!kBal) {
        if (h) {
#pragma unroll
            for (int k = 1; k < E; ++k) {
                float2 w = twN[k * E];  // W_2E^k = W_N^{k E}
                if (DIR > 0) w.y = -w.y;
                v[k] = cmul(v[k], w);
            }
        }
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float2 send = h ? v[i] : v[H + i];
            const float2 recv = make_float2(__shfl_xor_sync(0xffffffffu, send.x, NG),
                                            __shfl_xor_sync(0xffffffffu, send.y, NG));
            const float2 a = h ? recv : v[i];
            const float2 b = h ? v[H + i] : recv;
            v[i] = a + b;
            v[H + i] = a - b;
        }
        return;
    }
    const float2* tw2 = twN + h * H * E;  // W_2E^{h H + i} = tw2[i E]
#pragma unroll
    for (int i = 0; i < H; ++i) {
        const float2 send = v[H + i];  // h = 0: F0[H + i]; h = 1: F1[i]
        const float2 recv = make_float2(__shfl_xor_sync(0xffffffffu, send.x, NG),
                                        __shfl_xor_sync(0xffffffffu, send.y, NG));
        const float2 u = h ? v[i] : recv;  // F1[h H + i]
        const float2 o = h ? recv : v[i];  // F0[h H + i]
        float2 w = tw2[i * E];
        if (DIR > 0) w.y = -w.y;
        const float2 gk = cmul(u, w);
        v[i] = o + gk;      // X[h H + i]
        v[H + i] = o - gk;  // X[E + h H + i]
    }
}

template <int N, int E, int NG, int DIR, class Bar = BarCta, int PADX = 1>
__device__ __forceinline__ void fft_d3_to_d1(float2 (&v)[E], int t, int g, float2* xb, const float2* twN,
                                             const Bar& bar = Bar{}) {
    constexpr int P = 2 * E, H = E / 2;
    static_assert(P * E == N && (E & (E - 1)) == 0 && NG <= 16 && 32 % NG == 0, "shape");
    const int p = t >> 1, h = t & 1;
    // radix-2 split of the 2E-point transforms: A_k = X_k + X_{k+E}, B_k = (X_k - X_{k+E}) W_2E^k
    const float2* tw2 = twN + h * H * E;
#pragma unroll
    for (int i = 0; i < H; ++i) {
        const float2 a = v[i] + v[H + i];  // A_{h H + i}
        float2 w = tw2[i * E];
        if (DIR > 0) w.y = -w.y;
        const float2 b = cmul(v[i] - v[H + i], w);  // B_{h H + i}
        const float2 send = h ? a : b;
        const float2 recv = make_float2(__shfl_xor_sync(0xffffffffu, send.x, NG),
                                        __shfl_xor_sync(0xffffffffu, send.y, NG));
        v[i] = h ? b : a;  // h = 0: A_i, A_{H+i}; h = 1: B_{H+i}, B_i (rotated)
        v[H + i] = recv;
    }
    RF<E, DIR>::run(v);  // outputs t = 2m + h, times (-1)^m for h = 1
    bar.sync();
#pragma unroll
    for (int m = 0; m < E; ++m) xb[xslot3<N, E, NG, PADX>(p, 2 * m + h, g)] = v[m];
    bar.sync();
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) v[k1] = xb[xslot3<N, E, NG, PADX>(k1, t, g)];
    const float2* tw1 = d3_tw1<N>(twN, t);
    const float s0 = tw1[0].x;  // +-1
    v[0] = make_float2(v[0].x * s0, v[0].y * s0);
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) {
        float2 w = tw1[t * k1];  // t k1 < N: no wrap, a running index
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    RF<E, DIR>::run(v);
}

// k2 of register r of thread half h in distribution D3
template <int E> __device__ __forceinline__ int d3_k2(int r, int h) {
    return r < E / 2 ? h * (E / 2) + r : E + h * (E / 2) + (r - E / 2);
}
// Mode of register r of D3 thread (p, h) relative to p + h E^2/2: kz = p + h E^2/2 + d3_off(r).
template <int E> __device__ __forceinline__ constexpr int d3_off(int r) {
    return r < E / 2 ? E * r : E * E + E * (r - E / 2);
}
// Tiles of 8-byte values [row][g] (8 groups g per row) read in distribution D3 keep mode kz
// in row kz ^ ((kz / (E^2/2)) & 1): the two threads of a pair (one half-warp) hold modes
// E^2/2 apart, and the swapped parity puts them in opposite bank halves.  For the modes of
// D3 thread (p, h) the swapped bit is h: row = (p ^ h) + h E^2/2 + d3_off(r).  For D1
// (thread t, kz = t + 2E j) it is bit 0 of j / (E/4): row = (t ^ d1_flip(j)) + 2E j.
template <int E> __device__ __forceinline__ constexpr int d1_flip(int j) { return (j / (E / 4)) & 1; }

// Split / merge of a real FFT of length 2M done as an M-point complex FFT
// (z[m] = x[2m] + i x[2m+1]); w = W_2M^k = exp(-2 pi i k / 2M).
__device__ __forceinline__ float2 r2c_post_f(float2 zk, float2 zm, float2 w) {
    const float2 s = make_float2(zk.x + zm.x, zk.y - zm.y);
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);
    const float2 wd = cmul(w, d);
    return make_float2(0.5f * (s.x + wd.y), 0.5f * (s.y - wd.x));
}
__device__ __forceinline__ float2 c2r_pre_f(float2 xk, float2 xm, float2 w) {
    const float2 e = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 o = cmul(make_float2(xk.x - xm.x, xk.y + xm.y), cconj(w));
    return make_float2(e.x - o.y, e.y + o.x);
}

}  // namespace pfc
