// Register-resident single-dimension passes of the FP32 stepper (lengths 64, 96, 128, 160,
// 192, 256, 512, 1024).
//
//  k_ycol  complex FFT along y (either direction, optional scale) of a tile of TX
//          consecutive kx columns of one z-plane; in place or out of place.
//  k_xrow  the x pass on R consecutive rows of the mixed (kx, y, z) field: inverse real
//          FFT (nx/2-point complex FFT with the split/merge twiddles), the cubic term
//          of psi3_split.hpp:8-13 with stabilisation C (and the optional potential of
//          psi3_split.hpp:1-6), forward real FFT -- in place, one read and one write.
//
// A y pass, the x pass and a y pass replace the general y/x/y passes of the step;
// they stream whole tiles (contiguous rows for x, 64-byte column segments for y)
// and keep every FFT in registers with one shared-memory transpose per transform.
#include <cuda.h>
#include <cudaTypedefs.h>
#include "bulk.cuh"
#include "pfc_ctx.h"
#include "regfft.cuh"

namespace pfc {
namespace {

constexpr int cmaxi(int a, int b) { return a > b ? a : b; }

// Exchange padding of the four-step transforms of TX interleaved columns whose reads take
// U rows per thread: successive rows of a read are U (P TX) + U PADG slots apart, and
// with E even the 32 / TX thread groups of a warp land in alternate bank halves when
// U PADG = TX (mod 2 TX): PADG = TX / gcd(U, TX) (TX / U for powers of two).
constexpr int gcdi(int a, int b) { return b == 0 ? a : gcdi(b, a % b); }
constexpr int exch_pad(int tx, int u) { return tx / gcdi(u, tx); }

template <int NY_, int E_, int TX_, int MINB_ = 0>
struct YCfg {
    static constexpr int NY = NY_, E = E_, TX = TX_;
    static constexpr int P = NY / E, U = E / P, T = TX * P;
    static constexpr int PADG = TX < 32 ? exch_pad(TX, U) : 0;
    static constexpr int XB = E * (P * TX + PADG);
    static constexpr size_t SMEM = (size_t)(XB + NY) * sizeof(float2);
    static constexpr int MINB = MINB_ ? MINB_ : (T <= 128 ? 4 : 2);
    static_assert(P * E == NY && U * P == E && E % 2 == 0 && (TX >= 32 || 32 % TX == 0), "shape");
};

template <class Y, int DIR, bool kZ>
__global__ void __launch_bounds__(Y::T, Y::MINB)
    k_ycol(const float2* in, float2* out, int nxh, int ny, int nz, int lay, const float2* __restrict__ twg,
           float scale, int64_t ms, int q0, float2* copy) {
    // the columns of NY elements of kx tile blockIdx.x at plane q0 + blockIdx.y: y columns of
    // that z-plane (kZ false) or z columns at that ky (kZ); lay & 3: the layout of the input,
    // lay >> 2: of the output (col_addr).  With the standard layout on both sides, in may
    // equal out.  ms: elements between the fields of a batch (grid z).  copy (or null): the
    // input columns as read, written in the output's layout (a relayout fused with the FFT).
    constexpr int NY = Y::NY, E = Y::E, TX = Y::TX, P = Y::P, U = Y::U;
    in += blockIdx.z * ms;
    out += blockIdx.z * ms;
    extern __shared__ __align__(16) float2 sm[];
    float2* xb = sm;
    float2* tw = sm + Y::XB;
    const int tid = threadIdx.x;
    for (int i = tid; i < NY; i += Y::T) tw[i] = twg[i];
    const int c = tid % TX, t = tid / TX;
    const int kx = blockIdx.x * TX + c;
    const bool valid = kx < nxh;
    const int q = q0 + blockIdx.y;
    const ColAddr ai = col_addr(lay & 3, kZ, kx, q, nxh, ny, nz);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? in[ai.base + (int64_t)(t + P * j) * ai.stride] : make_float2(0.f, 0.f);
    if (copy && valid) {
        copy += blockIdx.z * ms;
        const ColAddr ac = col_addr(lay >> 2, kZ, kx, q, nxh, ny, nz);
#pragma unroll
        for (int j = 0; j < E; ++j) copy[ac.base + (int64_t)(t + P * j) * ac.stride] = v[j];
    }
    __syncthreads();
    fft_d1_to_d2<NY, E, TX, DIR, BarCta, Y::PADG>(v, t, c, xb, tw);
    if (valid) {
        const ColAddr ao = col_addr(lay >> 2, kZ, kx, q, nxh, ny, nz);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) {
                const float2 w = v[u * P + k2];
                out[ao.base + (int64_t)((t * U + u) + E * k2) * ao.stride] = make_float2(w.x * scale, w.y * scale);
            }
    }
}

// y columns of N = 2 E^2 points with E values per thread and 2E threads per column
// (fft_d1_to_d3): half the registers of YCfg's square split, so more resident warps.
template <int NY_, int E_, int TX_, int MINB_, bool BAL_>
struct YCfg3 {
    static constexpr int NY = NY_, E = E_, TX = TX_, P = 2 * E, T = TX * P, MINB = MINB_;
    static constexpr bool BAL = BAL_;                  // the balanced radix-2 step of fft_d1_to_d3
    static constexpr int TW = BAL ? 2 * NY : NY;       // its signed twiddle table, or W_NY^m alone
    static constexpr int XB = E * (P + 1) * TX;
    static constexpr size_t SMEM = (size_t)(XB + TW) * sizeof(float2);
    static_assert(P * E == NY && 32 % TX == 0, "shape");
};

// (lay as k_ycol: the layouts of in and out, y columns of z-plane blockIdx.y)
template <class Y, int DIR>
__global__ void __launch_bounds__(Y::T, Y::MINB)
    k_ycol3(const float2* in, float2* out, int nxh, int nz, int lay, const float2* __restrict__ twg, float scale,
            int64_t ms) {
    constexpr int NY = Y::NY, E = Y::E, TX = Y::TX, P = Y::P;
    in += blockIdx.z * ms;  // fields of a batch (grid z)
    out += blockIdx.z * ms;
    extern __shared__ __align__(16) float2 sm[];
    float2* xb = sm;
    float2* tw = sm + Y::XB;  // W_NY^m, then -W_NY^m (fft_d1_to_d3)
    const int tid = threadIdx.x;
    for (int i = tid; i < NY; i += Y::T) {
        const float2 w = twg[i];
        tw[i] = w;
        if (Y::BAL) tw[NY + i] = make_float2(-w.x, -w.y);
    }
    const int c = tid % TX, t = tid / TX;
    const int kx = blockIdx.x * TX + c;
    const bool valid = kx < nxh;
    const ColAddr ai = col_addr(lay & 3, false, kx, blockIdx.y, nxh, NY, nz);
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = valid ? in[ai.base + (int64_t)(t + P * j) * ai.stride] : make_float2(0.f, 0.f);
    __syncthreads();
    fft_d1_to_d3<NY, E, TX, DIR, BarCta, Y::BAL>(v, t, c, xb, tw);
    if (valid) {
        const ColAddr ao = col_addr(lay >> 2, false, kx, blockIdx.y, nxh, NY, nz);
        const int p = t >> 1, h = t & 1;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int k = p + E * d3_k2<E>(r, h);
            out[ao.base + (int64_t)k * ao.stride] = make_float2(v[r].x * scale, v[r].y * scale);
        }
    }
}

// The y pass between the two kx-tiled layouts with the TMA unit moving every whole tile:
// per CTA (kx tile kt, z-plane blockIdx.y) the 512 y values of the tile's TX columns are
// one contiguous 32 KB block in the row-tiled layout ([z][y][c]) and 512 pieces of 64
// bytes, nz TX elements apart, in the z-tiled layout ([ky][z][c]).  The row-tiled side
// moves by one 1-D bulk copy; the z-tiled side by tiled tensor copies of boxes of
// 16 x 1 x 256 floats over the map (floats of a tile row, z, ky, whole tile, field).  One
// elected thread arms the mbarrier and issues the loads; the stage then serves as the
// transform's exchange buffer and as the output stage, which one thread stores after a
// proxy fence.  The last, partial tile (nxh % TX columns) moves by per-thread accesses in
// the same launch.  LIN / LOUT: the layouts of in / out (1 z-tiled, 2 row-tiled).
template <class Y>
struct YBulkCfg {
    static constexpr int NY = Y::NY, TX = Y::TX;
    static constexpr int BOX = 256;                     // ky per tensor box (the box limit)
    static constexpr size_t SMEM = Y::SMEM + 16;        // exchange/stage, twiddles, mbarrier
    static_assert(Y::XB >= NY * TX && NY % BOX == 0 && TX == kTileW, "stage");
};

template <class Y, int DIR, int LIN, int LOUT>
__global__ void __launch_bounds__(Y::T, Y::MINB)
    k_ybulk(const float2* in, float2* out, int nxh, int nz, const __grid_constant__ CUtensorMap tmap,
            const float2* __restrict__ twg, float scale, int64_t ms, int* flag) {
    static_assert((LIN == 1 && LOUT == 2) || (LIN == 2 && LOUT == 1), "between the tiled layouts");
    using C = YBulkCfg<Y>;
    constexpr int NY = Y::NY, E = Y::E, TX = Y::TX, P = Y::P;
    constexpr unsigned kBlockBytes = NY * TX * sizeof(float2);
    in += blockIdx.z * ms;  // fields of a batch (grid z)
    out += blockIdx.z * ms;
    extern __shared__ __align__(128) float2 sm[];
    float2* xb = sm;
    float2* tw = sm + Y::XB;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tw + Y::TW);
    const int tid = threadIdx.x;
    const int c = tid % TX, t = tid / TX;
    const int kt = blockIdx.x, z = blockIdx.y;
    const bool whole = (kt + 1) * TX <= nxh;
    // the row-tiled block of (kt, z) (whole tiles)
    const int64_t rblk = ((int64_t)kt * nz + z) * (NY * TX);
    if (whole && tid == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
        mbar_arrive_expect_tx(bar, kBlockBytes);
        if (LIN == 2) bulk_load(xb, in + rblk, kBlockBytes, bar);
        else
#pragma unroll
            for (int h = 0; h < NY / C::BOX; ++h)
                tma_load5(xb + h * C::BOX * TX, &tmap, 0, z, h * C::BOX, kt, blockIdx.z, bar);
    }
    for (int i = tid; i < NY; i += Y::T) {
        const float2 w = twg[i];
        tw[i] = w;
        if (Y::BAL) tw[NY + i] = make_float2(-w.x, -w.y);
    }
    float2 v[E];
    const int kx = kt * TX + c;
    const bool valid = kx < nxh;
    if (!whole) {
        const ColAddr ai = col_addr(LIN, false, kx, z, nxh, NY, nz);
#pragma unroll
        for (int j = 0; j < E; ++j)
            v[j] = valid ? in[ai.base + (int64_t)(t + P * j) * ai.stride] : make_float2(0.f, 0.f);
    }
    __syncthreads();  // the twiddles, and the barrier's initialisation
    if (whole) {
        if (!mbar_wait(bar, 0, kWaitPolls)) {
            if (tid == 0) atomicOr(flag, kFlagWaitTimeout);
            return;
        }
#pragma unroll
        for (int j = 0; j < E; ++j) v[j] = xb[(t + P * j) * TX + c];
    }
    // (fft_d1_to_d3 synchronises before its first write to xb)
    fft_d1_to_d3<NY, E, TX, DIR, BarCta, Y::BAL>(v, t, c, xb, tw);
    const int p = t >> 1, h = t & 1;
    if (!whole) {
        if (valid) {
            const ColAddr ao = col_addr(LOUT, false, kx, z, nxh, NY, nz);
#pragma unroll
            for (int r = 0; r < E; ++r)
                out[ao.base + (int64_t)(p + E * d3_k2<E>(r, h)) * ao.stride] =
                    make_float2(v[r].x * scale, v[r].y * scale);
        }
        return;
    }
    __syncthreads();  // every thread's last exchange reads are done
#pragma unroll
    for (int r = 0; r < E; ++r) xb[(p + E * d3_k2<E>(r, h)) * TX + c] = make_float2(v[r].x * scale, v[r].y * scale);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        if (LOUT == 2) bulk_store(out + rblk, xb, kBlockBytes);
        else
#pragma unroll
            for (int h2 = 0; h2 < NY / C::BOX; ++h2)
                tma_store5(&tmap, xb + h2 * C::BOX * TX, 0, z, h2 * C::BOX, kt, blockIdx.z);
        bulk_commit();
        bulk_wait_read();  // shared memory stays valid until the stores have read it
    }
}

template <int NX_, int E_, int T_, int MINB_ = 0>
struct XCfg {
    static constexpr int NX = NX_, M = NX / 2, NXH = M + 1, E = E_, T = T_;
    static constexpr int P = M / E, U = E / P, R = T / P;
    static constexpr int LDR = NXH;  // odd: a warp over 32 rows at one k is conflict-free
    static constexpr int BUF = cmaxi(R * LDR, E * P * R);
    static constexpr size_t SMEM = (size_t)(BUF + M + M + 1) * sizeof(float2);
    static constexpr int MINB = MINB_ ? MINB_ : (E <= 16 ? 3 : 2);
    static_assert(P * E == M && U * P == E && (R % 32 == 0 || R == 16) && R * P == T, "shape");
};

// The R rows from row0 of a row-tiled field (k_xrow MODE 3) between global memory and the
// shared row buffer (row pitch LDR): kStore false loads, true stores.  Each tile holds the
// R rows as one contiguous block of R kTileW elements.  Eight lanes move one row's 64-byte
// piece (four whole pieces per warp access); the two rows of a half-warp are 8 apart, so
// with the odd pitch they fall in opposite halves of the shared-memory banks.
template <class X, bool kStore>
__device__ __forceinline__ void row_tiles(float2* rb, float2* g, int row0, int nrows, int tid) {
    constexpr int M = X::M, R = X::R, T = X::T, LDR = X::LDR, FT = M / kTileW;  // full tiles; the last: kx = M
    constexpr int CH = R * kTileW;  // elements of one tile's block of R rows
    static_assert(M % kTileW == 0 && kTileW == 8 && R % 16 == 0 && LDR % 2 == 1, "shape");
    static_assert(CH % T == 0 ? true : (T % CH == 0 && FT % (T / CH) == 0), "threads per tile block");
    constexpr int NPOS = CH >= T ? CH / T : 1;        // positions of a block per thread
    constexpr int TSTEP = CH >= T ? 1 : T / CH;       // tiles apart of a thread's blocks
    const int64_t ts = (int64_t)kTileW * nrows;       // elements between tiles
    const int kt0 = CH >= T ? 0 : tid / CH;
#pragma unroll
    for (int m = 0; m < NPOS; ++m) {
        const int pos = CH >= T ? tid + m * T : tid % CH;
        const int c = pos % kTileW, q = pos / kTileW, p = q >> 1;
        const int rr = (p & 7) + ((p >> 3) << 4) + ((q & 1) << 3);  // a bijection of [0, R)
        float2* gp = g + kt0 * ts + (int64_t)(row0 + rr) * kTileW + c;
        float2* sp = rb + rr * LDR + kt0 * kTileW + c;
#pragma unroll
        for (int k = 0; k < FT / TSTEP; ++k) {
            if (kStore) *gp = sp[k * TSTEP * kTileW];
            else sp[k * TSTEP * kTileW] = *gp;
            gp += TSTEP * ts;
        }
    }
    if (tid < R) {
        float2* gp = g + FT * ts + row0 + tid;
        float2* sp = rb + tid * LDR + M;
        if (kStore) *gp = *sp;
        else *sp = *gp;
    }
}

// The R2C merge of the x pass fused into the store of the R rows from row0 to a row-tiled
// field: rb holds y (the inverse transform's output, M per row); out[kx] =
// r2c_post_f(y[kx], y[(M - kx) mod M], W_NX^kx) for kx < M and out[M] = (Re y0 - Im y0, 0),
// in row_tiles's order (one shared-memory round trip fewer than merging in registers).
template <class X>
__device__ __forceinline__ void row_tiles_r2c(const float2* rb, const float2* twP, float2* g, int row0, int nrows,
                                              int tid) {
    constexpr int M = X::M, R = X::R, T = X::T, LDR = X::LDR, FT = M / kTileW;
    constexpr int CH = R * kTileW;
    static_assert(M % kTileW == 0 && kTileW == 8 && R % 16 == 0 && LDR % 2 == 1, "shape");
    constexpr int NPOS = CH >= T ? CH / T : 1;
    constexpr int TSTEP = CH >= T ? 1 : T / CH;
    const int64_t ts = (int64_t)kTileW * nrows;
    const int kt0 = CH >= T ? 0 : tid / CH;
#pragma unroll
    for (int m = 0; m < NPOS; ++m) {
        const int pos = CH >= T ? tid + m * T : tid % CH;
        const int c = pos % kTileW, q = pos / kTileW, p = q >> 1;
        const int rr = (p & 7) + ((p >> 3) << 4) + ((q & 1) << 3);
        float2* gp = g + kt0 * ts + (int64_t)(row0 + rr) * kTileW + c;
        const float2* row = rb + rr * LDR;
#pragma unroll
        for (int k = 0; k < FT / TSTEP; ++k) {
            const int kx = (kt0 + k * TSTEP) * kTileW + c;
            *gp = r2c_post_f(row[kx], row[kx == 0 ? 0 : M - kx], twP[kx]);  // Y[(M - kx) mod M]
            gp += TSTEP * ts;
        }
    }
    if (tid < R) {
        const float2 y0 = rb[tid * LDR];
        g[FT * ts + row0 + tid] = make_float2(y0.x - y0.y, 0.f);
    }
}

// MODE 0: the step's x pass, in place (in == out).  MODE 1: R2C of real rows (in: rows
// of M float2 pairs x[2m] + i x[2m+1]) into half-spectrum rows (out: rows of NXH).
// MODE 2: C2R of half-spectrum rows (in) into real rows (out, M pairs per row).  MODE 3:
// MODE 0 on the row-tiled layout (col_addr layout 2: element kx of row n = z ny + y at
// tile_base(kx / kTileW) + n wt + kx % kTileW, tile_base(kt) = kt kTileW nrows; nrows
// the field's rows, a multiple of R).  The transforms are unnormalised, as
// cufft_wrapper.hpp:61-86.
template <class X, int MODE>
__global__ void __launch_bounds__(X::T, X::MINB)
    k_xrow(const float2* in, float2* out, const float* __restrict__ pot, int nrows, const float2* __restrict__ twg,
           float mul, float Cc, float mu, int64_t ms) {
    constexpr int NX = X::NX, M = X::M, NXH = X::NXH, E = X::E, P = X::P, U = X::U, R = X::R, LDR = X::LDR;
    in += blockIdx.z * ms;  // fields of a batch (grid z; no potential then)
    out += blockIdx.z * ms;
    constexpr int LIN = MODE == 1 ? M : NXH;  // input row length (float2)
    extern __shared__ __align__(16) float2 sm[];
    float2* rb = sm;
    float2* twM = sm + X::BUF;  // W_M^m, m < M
    float2* twP = twM + M;      // W_NX^k, k <= M
    const int tid = threadIdx.x;
    for (int i = tid; i < 2 * M + 1; i += X::T) twM[i] = twg[i];
    const int r = tid % R, t = tid / R;
    const int row0 = blockIdx.x * R;
    const int nr = min(R, nrows - row0);
    const int64_t g0 = (int64_t)row0 * LIN;
    if constexpr (MODE == 3) {
        row_tiles<X, false>(rb, const_cast<float2*>(in), row0, nrows, tid);
    } else if constexpr (LIN == LDR) {
        for (int i = tid; i < nr * LIN; i += X::T) rb[i] = in[g0 + i];
    } else {
        for (int i = tid; i < nr * LIN; i += X::T) rb[(i / LIN) * LDR + i % LIN] = in[g0 + i];
    }
    __syncthreads();
    float2 v[E];
    if constexpr (MODE != 1) {
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int k = t + P * j;
            v[j] = c2r_pre_f(rb[r * LDR + k], rb[r * LDR + M - k], twP[k]);
        }
        fft_d1_to_d2<M, E, R, 1>(v, t, r, rb, twM);
    }
    if constexpr (MODE == 2) {
        // real pairs out through shared memory, so that rows are stored contiguously
        __syncthreads();
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) rb[r * LDR + (t * U + u) + E * k2] = v[u * P + k2];
        __syncthreads();
        for (int i = tid; i < nr * M; i += X::T) out[(int64_t)row0 * M + i] = rb[(i / M) * LDR + i % M];
        return;
    }
    if constexpr (MODE == 1) {
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) v[u * P + k2] = rb[r * LDR + (t * U + u) + E * k2];
    } else {
        const int64_t prow = (int64_t)(row0 + r) * NX;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k2 = 0; k2 < P; ++k2) {
                const int n = (t * U + u) + E * k2;
                const float2 x = v[u * P + k2];
                const float a = x.x * mul, b = x.y * mul;
                float2 o = make_float2(a * a * a - Cc * a - mu, b * b * b - Cc * b - mu);
                if (pot && r < nr) {
                    const float2 pp = *reinterpret_cast<const float2*>(pot + prow + 2 * n);
                    o.x += pp.x;
                    o.y += pp.y;
                }
                v[u * P + k2] = o;
            }
    }
    fft_d2_to_d1<M, E, R, -1>(v, t, r, rb, twM);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) rb[r * LDR + t + P * j] = v[j];
    __syncthreads();
    if constexpr (MODE == 3) {
        row_tiles_r2c<X>(rb, twP, out, row0, nrows, tid);
        return;
    }
    float2 xm_last = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int k = t + P * j;
        const float2 yk = v[j];
        if (k == 0) xm_last = make_float2(yk.x - yk.y, 0.f);  // X[nx/2]
        v[j] = r2c_post_f(yk, rb[r * LDR + (k == 0 ? 0 : M - k)], twP[k]);  // Y[(M - k) mod M]
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) rb[r * LDR + t + P * j] = v[j];
    if (t == 0) rb[r * LDR + M] = xm_last;
    __syncthreads();
    const int64_t o0 = (int64_t)row0 * NXH;
    for (int i = tid; i < nr * NXH; i += X::T) out[o0 + i] = rb[i];
}

// The x pass on row pairs (row-tiled layout, nx = 2 E^2 real points, e.g. 512 = 2 16^2):
// the two half-spectrum rows a, b of a pair make one full complex spectrum
// Z[k] = X_a[k] + i X_b[k] (X[nx - k] = conj X[k] for real rows), whose inverse FFT is
// x_a + i x_b; the cubic term of psi3_split.hpp:8-13 acts on real and imaginary parts;
// the forward FFT Z' of n_a + i n_b gives N_a[k] = (Z'[k] + conj Z'[nx - k]) / 2 and
// N_b[k] = (Z'[k] - conj Z'[nx - k]) / (2 i).  One nx-point complex FFT per pair and
// direction (fft_d1_to_d3 / fft_d3_to_d1: E values per thread, 2E threads per pair), no
// split or merge twiddles.  A CTA of 8 pairs (16 consecutive rows) holds its rows in
// shared memory interleaved by pair, [pair][kx][row of the pair], so that one 16-byte
// load gives both rows' mode kx.  Global traffic: the 16 rows of a tile are one
// contiguous 1 KB block of the row-tiled field; a warp moves 4 rows x 8 columns (256
// contiguous bytes) per access.
template <int NX_, int E_>
struct XPCfg {
    static constexpr int NX = NX_, E = E_, P = 2 * E, NG = 8, T = P * NG, R = 2 * NG;
    static constexpr int NXH = NX / 2 + 1;
    static constexpr int LDP = NXH;          // kx stride of a pair in the row stage (float4 units)
    static constexpr int LDZ = NX + 2;       // pair stride of the Z' stage (float2 units)
    static constexpr int XB = E * P * NG;    // exchange buffer (unpadded)
    static constexpr int BUF = cmaxi(cmaxi(NG * LDP * 2, XB), NG * LDZ);
    static constexpr int TW = 2 * NX;        // signed twiddles of fft_d1_to_d3
    static constexpr size_t SMEM = (size_t)(BUF + TW) * sizeof(float2);
    static_assert(P * E == NX && NX % (2 * kTileW) == 0, "shape");
};

template <class X>
__global__ void __launch_bounds__(X::T, 4) k_xpair(float2* g, int nrows, const float2* __restrict__ twg, float mul,
                                                   float Cc, float mu, int64_t ms) {
    constexpr int NX = X::NX, E = X::E, P = X::P, NG = X::NG, T = X::T, R = X::R, NXH = X::NXH;
    constexpr int FT = (NX / 2) / kTileW;  // whole tiles; the last tile holds kx = NX/2 alone
    extern __shared__ __align__(16) float2 sm[];
    float2* buf = sm;
    float2* tw = sm + X::BUF;
    float4* rows4 = reinterpret_cast<float4*>(buf);  // [pair][kx]: {row a, row b}
    const int tid = threadIdx.x;
    g += blockIdx.z * ms;  // fields of a batch (grid z)
    for (int i = tid; i < NX; i += T) {
        const float2 w = twg[i];
        tw[i] = w;
        tw[NX + i] = make_float2(-w.x, -w.y);
    }
    const int row0 = blockIdx.x * R;
    const int64_t ts = (int64_t)kTileW * nrows;  // elements between tiles
    const int lane = tid & 31, warp = tid >> 5, riw = lane >> 3, c = lane & 7;
    // load: unit u = (tile, group of 4 rows); a warp takes one unit per iteration
#pragma unroll 4
    for (int u = warp; u < FT * (R / 4); u += T / 32) {
        const int kt = u / (R / 4), rg = u % (R / 4);
        const int r = rg * 4 + riw;
        const float2 x = g[kt * ts + (int64_t)(row0 + r) * kTileW + c];
        buf[((r >> 1) * X::LDP + kt * kTileW + c) * 2 + (r & 1)] = x;
    }
    if (tid < R) buf[((tid >> 1) * X::LDP + NX / 2) * 2 + (tid & 1)] = g[FT * ts + row0 + tid];
    __syncthreads();
    // the pair's full spectrum Z in distribution D1 (thread t holds Z[t + P j])
    const int pg = tid % NG, t = tid / NG;
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
        const int k = t + P * j;
        const bool lo = k <= NX / 2;
        float4 ab = rows4[pg * X::LDP + (lo ? k : NX - k)];
        if (k == 0 || k == NX / 2) ab.y = ab.w = 0.f;  // real modes of real rows (as a C2R takes them)
        v[j] = lo ? make_float2(ab.x - ab.w, ab.y + ab.z) : make_float2(ab.x + ab.w, ab.z - ab.y);
    }
    // (fft_d1_to_d3 synchronises before it first writes the buffer)
    fft_d1_to_d3<NX, E, NG, 1, BarCta, true, 0>(v, t, pg, buf, tw);
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const float a = v[r].x * mul, b = v[r].y * mul;
        v[r] = make_float2(a * a * a - Cc * a - mu, b * b * b - Cc * b - mu);
    }
    fft_d3_to_d1<NX, E, NG, -1, BarCta, 0>(v, t, pg, buf, tw);
    __syncthreads();  // the last exchange reads are done
#pragma unroll
    for (int j = 0; j < E; ++j) buf[pg * X::LDZ + t + P * j] = v[j];
    __syncthreads();
    // store: lanes (pair of the warp's two, 16 consecutive kx); each writes both rows
    const int hp = lane >> 4, kk = lane & 15;
#pragma unroll 2
    for (int u = warp; u < (NG / 2) * (FT / 2); u += T / 32) {
        const int pp = 2 * (u % (NG / 2)) + hp, k = (u / (NG / 2)) * 16 + kk;
        const float2 z = buf[pp * X::LDZ + k], zm = buf[pp * X::LDZ + ((NX - k) & (NX - 1))];
        const float2 na = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
        const float2 nb = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        float2* gp = g + (k / kTileW) * ts + (int64_t)(row0 + 2 * pp) * kTileW + (k % kTileW);
        gp[0] = na;
        gp[kTileW] = nb;
    }
    if (tid < NG) {  // kx = NX/2 of both rows
        const float2 z = buf[tid * X::LDZ + NX / 2];
        g[FT * ts + row0 + 2 * tid] = make_float2(z.x, 0.f);
        g[FT * ts + row0 + 2 * tid + 1] = make_float2(z.y, 0.f);
    }
}

// The x pass with each row on one half-warp (row-tiled layout, nx = 2 P^2 real points with
// P = 16 lanes per row: 512).  Lane t of a row holds modes kx = t + P j (j < E = P), the
// four-step transforms' D1 = D2 distribution, so nothing is staged through shared memory
// but the transposes of the two transforms:
//  - load: the lane's modes straight from global memory; the split partner of mode kx,
//    nx/2 - kx, is register 15 - j of lane 16 - t (lane 0: its own register 16 - j, and
//    mode nx/2 itself), fetched by warp shuffle;
//  - C2R: c2r_pre_f, the nx/2-point inverse FFT (one transpose), cubic term, forward FFT
//    (one transpose), all exchanges within the half-warp (__syncwarp only);
//  - store: the R2C merge partner Y[(nx/2 - kx) mod nx/2] is register 15 - j of lane 16 - t
//    (lane 0: its own register (16 - j) mod 16), by warp shuffle; the merged modes go
//    straight to global memory.
// The split/merge twiddle W_nx^(t + P j) is W_nx^t (one table read per lane) times the
// compile-time constant W_(nx/P)^j.  Exchange slots of a row: (a, b) -> a (P + 1) + b, so
// both the writes (b = t) and the reads (a = t) of a half-warp fall on 16 distinct 8-byte
// bank pairs.  The stage twiddles W^{t k1} sit in a [k1][t] table (a half-warp reads 16
// consecutive entries).  A CTA holds 16 rows: one 1 KB block of each kx tile of the
// row-tiled field.
template <int NX_>
struct XLCfg {
    static constexpr int NX = NX_, M = NX / 2, P = 16, E = M / P, R = 16, T = R * P;
    static constexpr int LDA = P + 1, LDG = E * LDA;  // exchange: a stride, row stride
    static constexpr int XB = R * LDG;
    static constexpr size_t SMEM = (size_t)(XB + E * P) * sizeof(float2);
    static_assert(E == P && M % kTileW == 0 && P == 2 * kTileW, "shape");
};

template <class X>
__global__ void __launch_bounds__(X::T, 3) k_xlane(float2* g, int nrows, const float2* __restrict__ twg, float mul,
                                                   float Cc, float mu, int64_t ms) {
    constexpr int M = X::M, E = X::E, P = X::P, R = X::R, LDA = X::LDA, FT = M / kTileW;
    g += blockIdx.z * ms;  // fields of a batch (grid z)
    extern __shared__ __align__(16) float2 sm[];
    float2* tw2 = sm + X::XB;  // [k1][t]: W_M^{t k1}
    const int tid = threadIdx.x;
    for (int i = tid; i < E * P; i += X::T) tw2[i] = twg[(i % P) * (i / P)];
    const int t = tid % P, rl = tid / P;
    // the split/merge twiddle of mode t + P j: W_NX^t W_{NX/P}^j (the second a constant)
    const float2 wt = twg[M + t];
    float2* xr = sm + rl * X::LDG;
    const int64_t ts = (int64_t)kTileW * nrows;  // elements between tiles
    // row blocks in descending order: the y pass before this one wrote the last planes last,
    // so they are read while still in L2, and the first planes, which the y pass after this
    // one reads first, are written last
    const int blk = gridDim.x - 1 - blockIdx.x;
    const int64_t rowoff = (int64_t)(blk * R + rl) * kTileW;
    float2* gl = g + rowoff + (t & (kTileW - 1)) + (t / kTileW) * ts;  // mode t of the row
    float2* gnyq = g + FT * ts + blk * R + rl;                          // mode M (tile of width 1)
    const int src = (threadIdx.x & 31 & ~(P - 1)) | ((P - t) & (P - 1));  // the lane of mode M - t
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = gl[(2 * j) * ts];
    __syncthreads();
    // split: X[k] with X[M - k], which lane 16 - t holds at register 15 - j (lane 0: its own
    // register 16 - j, and X[M] for j = 0), register pairs (j, 15 - j) at a time; lane 0's
    // partner of register j is the original of register 16 - j, rewritten by the previous
    // pair, so it is carried over
    float2 carry = t == 0 ? *gnyq : make_float2(0.f, 0.f);
    sfor<0, E / 2>([&](auto jj) {
        constexpr int lo = decltype(jj)::value, hi = E - 1 - lo;
        const float2 vl = v[lo], vh = v[hi];
        float2 a = make_float2(__shfl_sync(0xffffffffu, vh.x, src), __shfl_sync(0xffffffffu, vh.y, src));
        float2 b = make_float2(__shfl_sync(0xffffffffu, vl.x, src), __shfl_sync(0xffffffffu, vl.y, src));
        if (t == 0) {
            a = carry;
            b = v[lo + 1];
        }
        carry = vh;
        v[lo] = c2r_pre_f(vl, a, twmul<X::NX / P, lo, -1>(wt));
        v[hi] = c2r_pre_f(vh, b, twmul<X::NX / P, hi, -1>(wt));
    });
    // inverse transform, D1 -> D2 (thread t: pair n = t + P k2 at register k2)
    RF<E, 1>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) {
        float2 w = tw2[k1 * P + t];
        w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) xr[k1 * LDA + t] = v[k1];
    __syncwarp();
#pragma unroll
    for (int tt = 0; tt < P; ++tt) v[tt] = xr[t * LDA + tt];
    RF<P, 1>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) {
        const float a = v[k2].x * mul, b = v[k2].y * mul;
        v[k2] = make_float2(a * a * a - Cc * a - mu, b * b * b - Cc * b - mu);
    }
    // forward transform, D2 -> D1
    RF<P, -1>::run(v);
#pragma unroll
    for (int k2 = 1; k2 < P; ++k2) v[k2] = cmul(v[k2], tw2[k2 * P + t]);
    __syncwarp();  // the first exchange's reads are done
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) xr[t * LDA + k2] = v[k2];
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < E; ++n1) v[n1] = xr[n1 * LDA + t];
    RF<E, -1>::run(v);
    // merge and store: Y[k] here, Y[(M - k) mod M] from lane 16 - t (lane 0: itself)
    sfor<0, E>([&](auto jj) {
        constexpr int j = decltype(jj)::value;
        const float2 s = v[E - 1 - j];
        float2 ym = make_float2(__shfl_sync(0xffffffffu, s.x, src), __shfl_sync(0xffffffffu, s.y, src));
        if (t == 0) ym = v[(E - j) & (E - 1)];
        gl[(2 * j) * ts] = r2c_post_f(v[j], ym, twmul<X::NX / P, j, -1>(wt));
    });
    if (t == 0) *gnyq = make_float2(v[0].x - v[0].y, 0.f);
}

template <class X>
cudaError_t xlattr() {
    return cudaFuncSetAttribute(k_xlane<X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
}
template <class X>
cudaError_t xllaunch(const pfc_ctx* c, void* b, double mul, double C, double mu, int nrows) {
    if (nrows % X::R) return cudaErrorNotSupported;
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->xpass_tw_off;
    k_xlane<X><<<dim3(nrows / X::R, 1, c->batch), X::T, X::SMEM, c->stream>>>((float2*)b, nrows, tw, (float)mul,
                                                                              (float)C, (float)mu, c->mstride);
    return cudaGetLastError();
}
using XL512 = XLCfg<512>;

using XP512 = XPCfg<512, 16>;
using XP128 = XPCfg<128, 8>;

template <class X>
cudaError_t xpattr() {
    return cudaFuncSetAttribute(k_xpair<X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
}
template <class X>
cudaError_t xplaunch(const pfc_ctx* c, void* b, double mul, double C, double mu, int nrows) {
    if (nrows % X::R) return cudaErrorNotSupported;
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->xpair_tw_off;
    k_xpair<X><<<dim3(nrows / X::R, 1, c->batch), X::T, X::SMEM, c->stream>>>((float2*)b, nrows, tw, (float)mul,
                                                                              (float)C, (float)mu, c->mstride);
    return cudaGetLastError();
}

using Y512 = YCfg<512, 32, 8>;              // z columns of the plain transforms (nz = 512)
using Y512q = YCfg3<512, 16, 8, 4, false>;  // the y pass: 16 values per thread, 64 registers

template <class Y>
cudaError_t y3attr() {
    cudaError_t e = cudaFuncSetAttribute(k_ycol3<Y, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y::SMEM);
    if (!e) e = cudaFuncSetAttribute(k_ycol3<Y, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y::SMEM);
    constexpr int kB = (int)YBulkCfg<Y>::SMEM;
    if (!e) e = cudaFuncSetAttribute(k_ybulk<Y, 1, 1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kB);
    if (!e) e = cudaFuncSetAttribute(k_ybulk<Y, -1, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kB);
    return e;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the
// driver library); null when the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The tensor map of the whole kx tiles of a z-tiled field (or batch of fields) at base:
// dimensions (the 2 kTileW floats of a tile row, z, ky, tile, field), boxes of
// 2 kTileW x 1 x box_ky x 1 x 1.  false when the shape has no such map (strides not
// multiples of 16 bytes, or no whole tile).
bool ztiled_map(const pfc_ctx* c, const void* base, int box_ky, CUtensorMap* m) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    const int full = c->nxh / kTileW;
    if (!enc || full < 1 || c->ny % box_ky) return false;
    const cuuint64_t row = kTileW * sizeof(float2);
    const cuuint64_t tile = row * (cuuint64_t)c->nz * (cuuint64_t)c->ny;
    const cuuint64_t field = c->batch > 1 ? (cuuint64_t)c->mstride * sizeof(float2) : tile * full;
    if (field % 16) return false;
    const cuuint64_t dims[5] = {2 * kTileW, (cuuint64_t)c->nz, (cuuint64_t)c->ny, (cuuint64_t)full,
                                (cuuint64_t)c->batch};
    const cuuint64_t strides[4] = {row, row * (cuuint64_t)c->nz, tile, field};
    const cuuint32_t box[5] = {2 * kTileW, 1, (cuuint32_t)box_ky, 1, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class Y>
cudaError_t y3launch(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int nzs, int lay) {
    dim3 grid((c->nxh + Y::TX - 1) / Y::TX, nzs, c->batch);
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->ypass_tw_off;
    // between the tiled layouts: the TMA kernel, the z-tiled side through a tensor map
    const bool inv_tiled = dir > 0 && lay == (1 | 2 << 2), fwd_tiled = dir < 0 && lay == (2 | 1 << 2);
    CUtensorMap m;
    if (c->ykern == 1 && (inv_tiled || fwd_tiled) &&
        ztiled_map(c, inv_tiled ? in : out, YBulkCfg<Y>::BOX, &m)) {
        constexpr size_t kB = YBulkCfg<Y>::SMEM;
        if (inv_tiled)
            k_ybulk<Y, 1, 1, 2><<<grid, Y::T, kB, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->nz, m, tw,
                                                              (float)scale, c->mstride, c->flag);
        else
            k_ybulk<Y, -1, 2, 1><<<grid, Y::T, kB, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->nz, m,
                                                               tw, (float)scale, c->mstride, c->flag);
        return cudaGetLastError();
    }
    if (dir > 0)
        k_ycol3<Y, 1><<<grid, Y::T, Y::SMEM, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->nz, lay, tw,
                                                          (float)scale, c->mstride);
    else
        k_ycol3<Y, -1><<<grid, Y::T, Y::SMEM, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->nz, lay, tw,
                                                           (float)scale, c->mstride);
    return cudaGetLastError();
}
using Y256 = YCfg<256, 16, 8>;
using Y128 = YCfg<128, 16, 8>;
using Y64 = YCfg<64, 8, 8>;
using X512h = XCfg<512, 16, 256>;  // 16 rows per CTA, 16 values per thread: three CTAs per SM
using X256 = XCfg<256, 16, 256>;
using X128 = XCfg<128, 16, 128>;
using X64 = XCfg<64, 8, 128>;
// 3 2^k lengths: 24 (or 12) values per thread over P = 8 or 4 threads per column or row,
// the first stage a radix-3 step (RF); small CTAs, so more of them per SM
using Y192 = YCfg<192, 24, 8, 12>;  // P 8, U 3: 64 threads, 80 registers
using Y96 = YCfg<96, 24, 8, 20>;   // P 4, U 6: 32 threads, 96 registers
using X192 = XCfg<192, 24, 128, 5>;  // M 96 = 24 x 4, 32 rows per CTA, 96 registers
using X96 = XCfg<96, 12, 128, 6>;   // M 48 = 12 x 4, 32 rows per CTA
// 5 2^k: 160 (the first stage a radix-5 step)
using Y160 = YCfg<160, 40, 8, 12>;  // P 4, U 10: 32 threads
using X160 = XCfg<160, 20, 128, 5>; // M 80 = 20 x 4, 32 rows per CTA
// 1024 (2D fields and y / x lengths beyond 512): 32 values per thread
using Y1024 = YCfg<1024, 32, 8>;     // P 32, U 1: 256 threads
using X1024 = XCfg<1024, 32, 256>;   // M 512 = 32 x 16, 16 rows per CTA

template <class Y, bool kZ>
cudaError_t yattr() {
    cudaError_t e =
        cudaFuncSetAttribute(k_ycol<Y, 1, kZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y::SMEM);
    if (e) return e;
    return cudaFuncSetAttribute(k_ycol<Y, -1, kZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y::SMEM);
}
template <class X>
cudaError_t xattr() {
    cudaError_t e = cudaFuncSetAttribute(k_xrow<X, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
    if (!e) e = cudaFuncSetAttribute(k_xrow<X, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
    if (!e) e = cudaFuncSetAttribute(k_xrow<X, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
    if (!e) e = cudaFuncSetAttribute(k_xrow<X, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)X::SMEM);
    return e;
}

// complex FFTs of the columns of the kx tiles of `planes` planes: z columns at each ky
// (kZ) or y columns of each z-plane; lay: the layouts of in / out (k_ycol); twiddles
// W_NY^m at tw_off
template <class Y, bool kZ>
cudaError_t collaunch(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int planes, int lay,
                      int tw_off, int q0 = 0, void* copy = nullptr) {
    dim3 grid((c->nxh + Y::TX - 1) / Y::TX, planes, c->batch);
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + tw_off;
    if (dir > 0)
        k_ycol<Y, 1, kZ><<<grid, Y::T, Y::SMEM, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->ny, c->nz,
                                                             lay, tw, (float)scale, c->mstride, q0, (float2*)copy);
    else
        k_ycol<Y, -1, kZ><<<grid, Y::T, Y::SMEM, c->stream>>>((const float2*)in, (float2*)out, c->nxh, c->ny, c->nz,
                                                              lay, tw, (float)scale, c->mstride, q0, (float2*)copy);
    return cudaGetLastError();
}
template <class Y>
cudaError_t ylaunch(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int nzs, int lay) {
    return collaunch<Y, false>(c, dir, in, out, scale, nzs, lay, c->ypass_tw_off);
}
template <class Y>
cudaError_t zlaunch_fft(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int lay, int ky0,
                        int nky, void* copy) {
    return collaunch<Y, true>(c, dir, in, out, scale, nky, lay, c->zfft_tw_off, ky0, copy);
}
template <class X, int MODE>
cudaError_t xlaunch(const pfc_ctx* c, const void* in, void* out, const void* pot, double mul, double C, double mu,
                    int nrows) {
    dim3 grid((nrows + X::R - 1) / X::R, 1, c->batch);
    const float2* tw = reinterpret_cast<const float2*>(c->tw) + c->xpass_tw_off;
    if (MODE == 3 && nrows % X::R) return cudaErrorNotSupported;  // whole tiles of rows
    if (pot && c->batch > 1) return cudaErrorNotSupported;
    k_xrow<X, MODE><<<grid, X::T, X::SMEM, c->stream>>>((const float2*)in, (float2*)out, (const float*)pot, nrows, tw,
                                                        (float)mul, (float)C, (float)mu, c->mstride);
    return cudaGetLastError();
}

}  // namespace

// Register y and x passes by length (0: none, the general passes run).  512 points: the y
// pass with 16 values per thread over 32 threads per column, capped at 64 registers
// (k_ycol3); the x pass with 16 values per thread, three CTAs per SM.
int fused_y_variant(int ny, int dtype) {
    if (dtype != PFC_F32) return 0;
    switch (ny) {
        case 512: return 7;
        case 256: return 2;
        case 128: return 3;
        case 64: return 4;
        case 192: return 10;
        case 96: return 11;
        case 160: return 12;
        case 1024: return 13;
    }
    return 0;
}
int fused_x_variant(int nx, int dtype) {
    if (dtype != PFC_F32) return 0;
    switch (nx) {
        case 512: return 5;
        case 256: return 2;
        case 128: return 3;
        case 64: return 4;
        case 192: return 10;
        case 96: return 11;
        case 160: return 12;
        case 1024: return 13;
    }
    return 0;
}

cudaError_t set_pass_attributes(const pfc_ctx* c) {
    cudaError_t e = cudaSuccess;
    switch (c->fused_y) {
        case 2: e = yattr<Y256, false>(); break;
        case 3: e = yattr<Y128, false>(); break;
        case 4: e = yattr<Y64, false>(); break;
        case 7: e = y3attr<Y512q>(); break;
        case 10: e = yattr<Y192, false>(); break;
        case 11: e = yattr<Y96, false>(); break;
        case 12: e = yattr<Y160, false>(); break;
        case 13: e = yattr<Y1024, false>(); break;
    }
    if (e) return e;
    switch (c->fused_x) {
        case 2: e = xattr<X256>(); break;
        case 3: e = xattr<X128>(); break;
        case 4: e = xattr<X64>(); break;
        case 5: e = xattr<X512h>(); break;
        case 10: e = xattr<X192>(); break;
        case 11: e = xattr<X96>(); break;
        case 12: e = xattr<X160>(); break;
        case 13: e = xattr<X1024>(); break;
    }
    if (!e && c->xkern == 1) e = c->nx == 512 ? xpattr<XP512>() : xpattr<XP128>();
    if (!e && c->xkern == 2) e = xlattr<XL512>();
    return e;
}

bool ybulk_available(const pfc_ctx* c) { return c->fused_y == 7 && tmap_encoder() != nullptr; }

cudaError_t launch_ypass(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int nzs, int lay) {
    if (lay && nzs != c->nz) return cudaErrorNotSupported;  // tiled: whole fields
    switch (c->fused_y) {
        case 2: return ylaunch<Y256>(c, dir, in, out, scale, nzs, lay);
        case 3: return ylaunch<Y128>(c, dir, in, out, scale, nzs, lay);
        case 4: return ylaunch<Y64>(c, dir, in, out, scale, nzs, lay);
        case 7: return y3launch<Y512q>(c, dir, in, out, scale, nzs, lay);
        case 10: return ylaunch<Y192>(c, dir, in, out, scale, nzs, lay);
        case 11: return ylaunch<Y96>(c, dir, in, out, scale, nzs, lay);
        case 12: return ylaunch<Y160>(c, dir, in, out, scale, nzs, lay);
        case 13: return ylaunch<Y1024>(c, dir, in, out, scale, nzs, lay);
    }
    return cudaErrorNotSupported;
}

template <int MODE>
cudaError_t xdispatch(const pfc_ctx* c, const void* in, void* out, const void* pot, double mul, double C, double mu,
                      int nrows) {
    switch (c->fused_x) {
        case 2: return xlaunch<X256, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 3: return xlaunch<X128, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 4: return xlaunch<X64, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 5: return xlaunch<X512h, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 10: return xlaunch<X192, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 11: return xlaunch<X96, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 12: return xlaunch<X160, MODE>(c, in, out, pot, mul, C, mu, nrows);
        case 13: return xlaunch<X1024, MODE>(c, in, out, pot, mul, C, mu, nrows);
    }
    return cudaErrorNotSupported;
}

cudaError_t launch_xpass(const pfc_ctx* c, void* b, const void* pot, double mul, double C, double mu, int nzs,
                         int lay) {
    if (lay == 2 && nzs != c->nz) return cudaErrorNotSupported;
    if (lay == 2 && !pot && c->xkern == 1) {
        switch (c->nx) {
            case 512: return xplaunch<XP512>(c, b, mul, C, mu, nzs * c->ny);
            case 128: return xplaunch<XP128>(c, b, mul, C, mu, nzs * c->ny);
        }
    }
    if (lay == 2 && !pot && c->xkern == 2 && c->nx == 512) return xllaunch<XL512>(c, b, mul, C, mu, nzs * c->ny);
    if (lay == 2) return xdispatch<3>(c, b, b, pot, mul, C, mu, nzs * c->ny);
    if (lay != 0) return cudaErrorNotSupported;
    return xdispatch<0>(c, b, b, pot, mul, C, mu, nzs * c->ny);
}
cudaError_t launch_xrows_r2c(const pfc_ctx* c, const void* in_real, void* out_cmpl) {
    return xdispatch<1>(c, in_real, out_cmpl, nullptr, 1.0, 0.0, 0.0, c->ny * c->nz);
}
cudaError_t launch_xrows_c2r(const pfc_ctx* c, const void* in_cmpl, void* out_real) {
    return xdispatch<2>(c, in_cmpl, out_real, nullptr, 1.0, 0.0, 0.0, c->ny * c->nz);
}

int fused_zfft_variant(int nz, int dtype) {
    if (dtype != PFC_F32) return 0;
    switch (nz) {
        case 512: return 1;
        case 256: return 2;
        case 128: return 3;
        case 64: return 4;
        case 192: return 10;
        case 96: return 11;
        case 160: return 12;
    }
    return 0;
}
cudaError_t set_zfft_attributes(const pfc_ctx* c) {
    switch (c->fused_zfft) {
        case 1: return yattr<Y512, true>();
        case 2: return yattr<Y256, true>();
        case 3: return yattr<Y128, true>();
        case 4: return yattr<Y64, true>();
        case 10: return yattr<Y192, true>();
        case 11: return yattr<Y96, true>();
        case 12: return yattr<Y160, true>();
    }
    return cudaSuccess;
}
// the packed row-pair x pass exists for nx = 2 E^2 (128 and 512), the row per half-warp for 512
int xkernel_variants(int nx, int dtype) {
    if (dtype != PFC_F32) return 1;
    return 1 | (nx == 512 || nx == 128 ? 2 : 0) | (nx == 512 ? 4 : 0);
}
// k_xlane where the length has it (512: 0.288 against 0.338 ms for k_xrow and 0.348 for
// k_xpair per 512^3 pass), else k_xrow
int default_xkernel(int variants) { return (variants & 4) ? 2 : 0; }

cudaError_t launch_zfft(const pfc_ctx* c, int dir, const void* in, void* out, double scale, int lay, int ky0,
                        int nky, void* copy) {
    if (nky < 0) nky = c->ny - ky0;
    if (ky0 < 0 || nky < 1 || ky0 + nky > c->ny) return cudaErrorInvalidValue;
    switch (c->fused_zfft) {
        case 1: return zlaunch_fft<Y512>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 2: return zlaunch_fft<Y256>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 3: return zlaunch_fft<Y128>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 4: return zlaunch_fft<Y64>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 10: return zlaunch_fft<Y192>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 11: return zlaunch_fft<Y96>(c, dir, in, out, scale, lay, ky0, nky, copy);
        case 12: return zlaunch_fft<Y160>(c, dir, in, out, scale, lay, ky0, nky, copy);
    }
    return cudaErrorNotSupported;
}

}  // namespace pfc
