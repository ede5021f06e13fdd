// Local-maximum peak finding (cuda/kernels/findpeaks.hpp:7-29, findpeaks_2d.hpp:7-27).
// A cell is a peak when it is strictly greater than all 26 (3D) or 8 (2D) periodic
// neighbours and >= ths.  Output sorted by linear index (deterministic).
//
// Two implementations: the context's (k_peaks_mark ... k_peaks_emit below: the stencil once
// per cell in shared memory, a bit mask, a compaction of the bits), and the one of the
// entry point without allocation, whose scratch must stay small (pass 1 counts peaks per
// block of kPeakBlock consecutive cells, one block scans the counts, pass 2 evaluates the
// stencil again and writes each peak at block offset + warp-ballot rank).
#include <cuda.h>
#include <cstdio>
#include <mutex>
#include "pfc_ctx.h"
#include <type_traits>

namespace pfc {
namespace {

template <typename T> struct MaxRec;
template <> struct MaxRec<float> { float i0, i1, i2; float field; };
template <> struct MaxRec<double> { double i0, i1, i2; float field; float pad; };  // pad written as 0
static_assert(sizeof(MaxRec<float>) == 16, "Maximum<float> layout");
static_assert(sizeof(MaxRec<double>) == 32, "Maximum<double> layout");

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

template <typename T>
__device__ __forceinline__ bool peak_at(const T* __restrict__ psi, int64_t idx, int nx, int ny, int nz, bool d3,
                                        T ths) {
    const int i0 = (int)(idx % nx);
    const int64_t r = idx / nx;
    const int i1 = (int)(r % ny), i2 = (int)(r / ny);
    const T v = psi[idx];
    bool ok = true;
    const int zlo = d3 ? -1 : 0, zhi = d3 ? 1 : 0;
    for (int dz = zlo; dz <= zhi; ++dz) {
        const int j2 = d3 ? wrapi(i2 + dz, nz) : i2;
        for (int dy = -1; dy <= 1; ++dy) {
            const int j1 = wrapi(i1 + dy, ny);
            const int64_t rowb = ((int64_t)j2 * ny + j1) * nx;
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                ok &= (v > psi[rowb + wrapi(i0 + dx, nx)]);
            }
        }
    }
    return ok && (v >= ths);
}

template <typename T>
__global__ void __launch_bounds__(kPeakBlock) k_peaks_count(const T* __restrict__ psi, int nx, int ny, int nz, int d3,
                                                            T ths, int* __restrict__ counts) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t idx = (int64_t)blockIdx.x * kPeakBlock + threadIdx.x;
    const bool f = idx < n && peak_at<T>(psi, idx, nx, ny, nz, d3 != 0, ths);
    const int c = __syncthreads_count(f);
    if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// Exclusive scan of nb counts by one block of 1024 threads; offsets[nb] = total.
__global__ void __launch_bounds__(1024) k_scan(const int* __restrict__ counts, int nb, int* __restrict__ offsets) {
    __shared__ int part[1024];
    const int chunk = (nb + 1023) / 1024;
    const int b = threadIdx.x * chunk;
    const int e = min(nb, b + chunk);
    int s = 0;
    for (int i = b; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = part[threadIdx.x] - s;
    for (int i = b; i < e; ++i) { offsets[i] = run; run += counts[i]; }
    if (threadIdx.x == 1023) offsets[nb] = part[1023];
}

template <typename T>
__global__ void __launch_bounds__(kPeakBlock) k_peaks_write(const T* __restrict__ psi, int nx, int ny, int nz, int d3,
                                                            T ths, const int* __restrict__ offsets,
                                                            MaxRec<T>* __restrict__ out, int capacity) {
    __shared__ int wsum[kPeakBlock / 32];
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t idx = (int64_t)blockIdx.x * kPeakBlock + threadIdx.x;
    const bool f = idx < n && peak_at<T>(psi, idx, nx, ny, nz, d3 != 0, ths);
    const unsigned m = __ballot_sync(0xffffffffu, f);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    if (!f) return;
    int pos = offsets[blockIdx.x] + __popc(m & ((1u << lane) - 1u));
    for (int w = 0; w < warp; ++w) pos += wsum[w];
    if (pos >= capacity) return;
    const int i0 = (int)(idx % nx);
    const int64_t r = idx / nx;
    MaxRec<T> rec = {};
    rec.i0 = (T)i0;
    rec.i1 = (T)(int)(r % ny);
    rec.i2 = (T)(int)(r / ny);
    rec.field = (float)psi[idx];
    out[pos] = rec;
}

// counts: one int per kPeakBlock cells; offsets: their exclusive scan plus the total
template <typename T>
cudaError_t peaks_raw(const void* psi, int nx, int ny, int nz, double ths, int* counts, int* offsets, void* out,
                      int capacity, cudaStream_t st) {
    const int d3 = nz > 1 ? 1 : 0;
    const int nb = (int)(((int64_t)nx * ny * nz + kPeakBlock - 1) / kPeakBlock);
    k_peaks_count<T><<<nb, kPeakBlock, 0, st>>>((const T*)psi, nx, ny, nz, d3, (T)ths, counts);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    k_scan<<<1, 1024, 0, st>>>(counts, nb, offsets);
    if ((e = cudaGetLastError())) return e;
    if (capacity > 0 && out) {
        k_peaks_write<T><<<nb, kPeakBlock, 0, st>>>((const T*)psi, nx, ny, nz, d3, (T)ths, offsets, (MaxRec<T>*)out,
                                                    capacity);
        if ((e = cudaGetLastError())) return e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------------------
// The context's peak finder: the stencil is evaluated once per cell, in shared memory, and
// leaves one bit per cell; the compaction then reads only the bits.
//
//  k_peaks_mark   a CTA of 32 x 8 threads owns a tile of 32 x 8 cells of kZC consecutive
//                 z-planes.  Plane by plane (with one halo plane below and above) it stages
//                 the tile and its periodic halo, 34 x 10 values, in shared memory; each
//                 thread forms the maximum M9 of its 3 x 3 in-plane neighbourhood and the
//                 maximum N8 of the 8 in-plane neighbours.  A cell of plane z is a peak when
//                 psi > max(M9(z-1), N8(z), M9(z+1)) (26 neighbours; 2D: N8 alone) and
//                 psi >= ths.  The maxima propagate NaN, so a NaN anywhere in the
//                 neighbourhood makes the strict comparison false, exactly as the 26
//                 comparisons of the reference (findpeaks.hpp:7-29, findpeaks_2d.hpp:7-27).
//                 Bit x % 32 of word (z, y, x / 32) is the cell (x, y, z): one warp ballot
//                 per row segment.
//  k_words_count  per chunk of kChunkWords words (eight warps of 1024 consecutive words, one
//                 word per lane and iteration): the number of set bits.
//  k_scan         (above) exclusive scan of the chunk counts.
//  k_peaks_emit   per chunk: the warps' bit counts, then per iteration a warp scan of the
//                 32 words' counts and one record per set bit at its rank -- in
//                 linear-index order.
// ---------------------------------------------------------------------------------------
constexpr int kTX = 32, kTY = 8, kZC = 16;
constexpr int kChunkWords = 256 * 32;

__device__ __forceinline__ float nmax(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }

template <typename T, bool D3>
__global__ void __launch_bounds__(kTX * kTY) k_peaks_mark(const T* __restrict__ psi, int nx, int ny, int nz, T ths,
                                                          uint32_t* __restrict__ mask, int wpr) {
    __shared__ T S[kTY + 2][kTX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int z0 = D3 ? blockIdx.z * kZC : 0;
    const int zend = D3 ? min(z0 + kZC, nz) : 1;
    const int x = x0 + tx, y = y0 + ty;
    const bool inside = x < nx && y < ny;
    // the tile and its halo, (kTY + 2)(kTX + 2) = 340 values: at most two per thread, at
    // in-plane offsets fixed for every plane (periodic wrap done once).  Cells of a partial
    // tile past the grid's edge only fill the tile (no cell inside reads them): offset -1.
    constexpr int kHalo = (kTY + 2) * (kTX + 2);
    int off[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int i = tid + m * kTX * kTY;
        off[m] = -1;
        if (i < kHalo) {
            const int r = i / (kTX + 2), q = i - r * (kTX + 2);
            int gy = y0 + r - 1, gx = x0 + q - 1;
            gy = gy < 0 ? gy + ny : (gy >= ny ? gy - ny : gy);
            gx = gx < 0 ? gx + nx : (gx >= nx ? gx - nx : gx);
            if (gy < ny && gx < nx) off[m] = gy * nx + gx;
        }
    }
    T* Sf = &S[0][0];
    // Planes are loaded kAhead planes ahead of their use into registers, so that the loads of
    // later planes are in flight while a plane is compared (the plane loop is otherwise a
    // chain of load latencies and barriers).
    constexpr int kAhead = 4;
    T ring[kAhead][2];
    auto load = [&](int zp, T (&dst)[2]) {
        const int zz = D3 ? (zp < 0 ? zp + nz : (zp >= nz ? zp - nz : zp)) : 0;
        const T* plane = psi + (int64_t)zz * ny * nx;
#pragma unroll
        for (int m = 0; m < 2; ++m) dst[m] = off[m] >= 0 ? plane[off[m]] : T(0);
    };
    T m9_prev = T(0), m9_cur = T(0), n8_cur = T(0), v_cur = T(0);
    const int zfirst = D3 ? z0 - 1 : 0, zlast = D3 ? zend : 0;
#pragma unroll
    for (int a = 0; a < kAhead; ++a)
        if (zfirst + a <= zlast) load(zfirst + a, ring[a]);
    for (int zp = zfirst; zp <= zlast; ++zp) {
        const int slot = (zp - zfirst) % kAhead;
        __syncthreads();  // the previous plane's reads are done
        T cur[2];
#pragma unroll
        for (int a = 0; a < kAhead; ++a)
            if (a == slot) {
                cur[0] = ring[a][0];
                cur[1] = ring[a][1];
                if (zp + kAhead <= zlast) load(zp + kAhead, ring[a]);
            }
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int i = tid + m * kTX * kTY;
            if (i < kHalo) Sf[i] = cur[m];
        }
        __syncthreads();
        const T r0 = nmax(nmax(S[ty][tx], S[ty][tx + 1]), S[ty][tx + 2]);
        const T r2 = nmax(nmax(S[ty + 2][tx], S[ty + 2][tx + 1]), S[ty + 2][tx + 2]);
        const T v = S[ty + 1][tx + 1];
        const T n8 = nmax(nmax(r0, r2), nmax(S[ty + 1][tx], S[ty + 1][tx + 2]));
        const T m9 = nmax(n8, v);
        if (D3 && zp >= z0 + 1) {
            // the cell of plane zp - 1 has all of its neighbours: M9(zp - 2), N8(zp - 1), M9(zp)
            const T m = nmax(nmax(m9_prev, n8_cur), m9);
            const bool pk = inside && v_cur > m && v_cur >= ths;
            const unsigned b = __ballot_sync(0xffffffffu, pk);
            if (tx == 0 && y < ny) mask[((int64_t)(zp - 1) * ny + y) * wpr + blockIdx.x] = b;
        }
        if (!D3) {
            const bool pk = inside && v > n8 && v >= ths;
            const unsigned b = __ballot_sync(0xffffffffu, pk);
            if (tx == 0 && y < ny) mask[(int64_t)y * wpr + blockIdx.x] = b;
        }
        m9_prev = m9_cur;
        m9_cur = m9;
        n8_cur = n8;
        v_cur = v;
    }
}

// The same stencil for FP32 3D fields with nx a multiple of 128 and ny of 16, at fewer
// instructions per cell: a CTA of 18 warps owns 128 x 16 cells of kZC4 consecutive planes.
// Warp w holds row y0 + w - 1 (w = 0 and 17 are the periodic halo rows), lane L the four
// cells x0 + 4L .. 4L + 3.  Planes stream through a ring of kStages4 slots in shared memory
// by cp.async (each lane copies its own 16 bytes, lanes 0 and 31 also the cell beyond the
// warp's edge, and reads back only what it copied: no barrier for the ring), kStages4 - 1
// planes ahead of their use.  In a plane each lane forms, per cell, lr = max of its two x
// neighbours (the outer ones by warp shuffle) and h = max(left, psi, right); h goes to shared
// memory (double-buffered, one barrier per plane), and the interior warps read the rows above
// and below: M9 = max(h(y-1), h, h(y+1)), N8 = max(h(y-1), h(y+1), lr).  The maxima of three
// are one instruction each (nmax3).  The 3D test and the NaN semantics are k_peaks_mark's.
// The four bits of a lane are OR-ed over the eight lanes of a mask word by three shuffles.
// Measured at 512^3 on a B200: issue-bound (ALU pipe 60%, 240 M warp instructions), not
// bandwidth-bound.
constexpr int kZC4 = 32, kRows4 = 16, kStages4 = 8;
// dynamic shared memory of k_peaks_mark4: the ring, the h rows, the edge cells
constexpr size_t kMark4Smem = (size_t)(kStages4 + 2) * (kRows4 + 2) * 32 * sizeof(float4) +
                              (size_t)kStages4 * (kRows4 + 2) * 2 * sizeof(float);

__device__ __forceinline__ float4 nmax4(float4 a, float4 b) {
    return make_float4(nmax(a.x, b.x), nmax(a.y, b.y), nmax(a.z, b.z), nmax(a.w, b.w));
}
// the NaN-propagating maximum of three (the three-input form of max.NaN.f32, sm_100)
__device__ __forceinline__ float nmax3(float a, float b, float c) {
    float r;
    asm("max.NaN.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float4 nmax34(float4 a, float4 b, float4 c) {
    return make_float4(nmax3(a.x, b.x, c.x), nmax3(a.y, b.y, c.y), nmax3(a.z, b.z, c.z), nmax3(a.w, b.w, c.w));
}
__device__ __forceinline__ void cp_async16_cg(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(32 * (kRows4 + 2), 2)
    k_peaks_mark4(const float* __restrict__ psi, int nx, int ny, int nz, float ths, uint32_t* __restrict__ mask,
                  int wpr) {
    extern __shared__ __align__(16) float4 sm4[];
    float4 (*H)[kRows4 + 2][32] = reinterpret_cast<float4 (*)[kRows4 + 2][32]>(sm4);
    float4 (*Q)[kRows4 + 2][32] = reinterpret_cast<float4 (*)[kRows4 + 2][32]>(sm4 + 2 * (kRows4 + 2) * 32);
    float (*EG)[kRows4 + 2][2] =
        reinterpret_cast<float (*)[kRows4 + 2][2]>(sm4 + (kStages4 + 2) * (kRows4 + 2) * 32);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x0 = blockIdx.x * 128, y0 = blockIdx.y * kRows4, z0 = blockIdx.z * kZC4;
    const int zend = min(z0 + kZC4, nz);
    int y = y0 + w - 1;
    y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
    const float* rowp = psi + (int64_t)y * nx + x0 + 4 * lane;  // the lane's cells in plane 0
    // the edge cell of lanes 0 and 31, relative to rowp (periodic in x)
    const bool edge = lane == 0 || lane == 31;
    const int eoff = lane == 0 ? (x0 == 0 ? nx - 1 : -1) : (x0 + 128 == nx ? -x0 - 124 : 4);
    float* eslot = &EG[0][w][lane == 0 ? 0 : 1];
    const int64_t plane = (int64_t)ny * nx;
    const int zfirst = z0 - 1, zlast = zend;
    auto issue = [&](int zp) {
        if (zp <= zlast) {
            const int zz = zp < 0 ? zp + nz : (zp >= nz ? zp - nz : zp);
            const float* p = rowp + zz * plane;
            const int s = (zp - zfirst) % kStages4;
            cp_async16_cg(&Q[s][w][lane], p);
            if (edge) cp_async4(eslot + s * (kRows4 + 2) * 2, p + eoff);
        }
        cp_commit_group();  // (empty past the last plane: the group count stays regular)
    };
#pragma unroll
    for (int s = 0; s < kStages4 - 1; ++s) issue(zfirst + s);
    const bool interior = w >= 1 && w <= kRows4;
    float4 m9p = make_float4(0.f, 0.f, 0.f, 0.f), m9c = m9p, n8c = m9p, vc = m9p;
    for (int zp = zfirst; zp <= zlast; ++zp) {
        issue(zp + kStages4 - 1);  // into the slot of plane zp - 1, which this thread has read
        cp_wait_group<kStages4 - 1>();
        const int s = (zp - zfirst) % kStages4;
        const float4 q = Q[s][w][lane];
        const float e = edge ? eslot[s * (kRows4 + 2) * 2] : 0.f;
        float left = __shfl_up_sync(0xffffffffu, q.w, 1), right = __shfl_down_sync(0xffffffffu, q.x, 1);
        if (lane == 0) left = e;
        if (lane == 31) right = e;
        const float4 lr = make_float4(nmax(left, q.y), nmax(q.x, q.z), nmax(q.y, q.w), nmax(q.z, right));
        const float4 h = make_float4(nmax3(left, q.x, q.y), nmax3(q.x, q.y, q.z), nmax3(q.y, q.z, q.w),
                                     nmax3(q.z, q.w, right));
        const int buf = (zp - zfirst) & 1;
        H[buf][w][lane] = h;
        __syncthreads();
        if (interior) {
            const float4 up = H[buf][w - 1][lane], dn = H[buf][w + 1][lane];
            const float4 m9 = nmax34(up, h, dn), n8 = nmax34(up, dn, lr);
            if (zp >= z0 + 1) {
                // the cells of plane zp - 1: M9(zp - 2), N8(zp - 1), M9(zp)
                const float4 m = nmax34(m9p, n8c, m9);
                uint32_t nib = (vc.x > m.x && vc.x >= ths ? 1u : 0u) | (vc.y > m.y && vc.y >= ths ? 2u : 0u) |
                               (vc.z > m.z && vc.z >= ths ? 4u : 0u) | (vc.w > m.w && vc.w >= ths ? 8u : 0u);
                nib <<= 4 * (lane & 7);
                nib |= __shfl_xor_sync(0xffffffffu, nib, 1);
                nib |= __shfl_xor_sync(0xffffffffu, nib, 2);
                nib |= __shfl_xor_sync(0xffffffffu, nib, 4);
                if ((lane & 7) == 0) mask[((int64_t)(zp - 1) * ny + y) * wpr + (x0 >> 5) + (lane >> 3)] = nib;
            }
            m9p = m9c;
            m9c = m9;
            n8c = n8;
            vc = q;
        }
    }
    cp_wait_group<0>();
}

// A chunk of kChunkWords mask words per block: warp w takes words [w 1024, (w + 1) 1024) of
// the chunk, 32 consecutive words (one per lane) per iteration -- coalesced.
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}
__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(256) k_words_count(const uint32_t* __restrict__ mask, int64_t nwords,
                                                     int* __restrict__ counts) {
    __shared__ int ws[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t w0 = (int64_t)blockIdx.x * kChunkWords + warp * 1024 + lane;
    int c = 0;
#pragma unroll
    for (int it = 0; it < 32; ++it) {
        const int64_t w = w0 + it * 32;
        if (w < nwords) c += __popc(mask[w]);
    }
    c = warp_sum(c);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < 8; ++i) t += ws[i];
        counts[blockIdx.x] = t;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_peaks_emit(const T* __restrict__ psi, const uint32_t* __restrict__ mask,
                                                    int64_t nwords, int nx, int ny, int wpr,
                                                    const int* __restrict__ offsets, MaxRec<T>* __restrict__ out,
                                                    int capacity) {
    __shared__ int ws[8];
    __shared__ uint32_t words[8][32][32];  // the warps' words, kept for the emit pass
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t w0 = (int64_t)blockIdx.x * kChunkWords + warp * 1024 + lane;
    // the warp's 1024 words, all loads in flight at once
    uint32_t wv[32];
#pragma unroll
    for (int it = 0; it < 32; ++it) {
        const int64_t w = w0 + it * 32;
        wv[it] = w < nwords ? mask[w] : 0u;
    }
    int c = 0;
#pragma unroll
    for (int it = 0; it < 32; ++it) {
        c += __popc(wv[it]);
        words[warp][it][lane] = wv[it];
    }
    c = warp_sum(c);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    if (c == 0) return;  // (warp-uniform)
    int base = offsets[blockIdx.x];
    for (int w = 0; w < warp; ++w) base += ws[w];
    for (int it = 0; it < 32; ++it) {
        const int64_t w = w0 + it * 32;
        const uint32_t word = words[warp][it][lane];
        const int n = __popc(word);
        const int incl = warp_incl_scan(n, lane);
        int pos = base + incl - n;
        base += __shfl_sync(0xffffffffu, incl, 31);
        uint32_t b = word;
        if (b) {
            const int64_t row = w / wpr;
            const int xb = (int)(w - row * wpr) * 32;
            while (b) {
                const int bit = __ffs(b) - 1;
                b &= b - 1;
                if (pos < capacity) {
                    const int xx = xb + bit;
                    MaxRec<T> rec = {};
                    rec.i0 = (T)xx;
                    rec.i1 = (T)(int)(row % ny);
                    rec.i2 = (T)(int)(row / ny);
                    rec.field = (float)psi[row * nx + xx];
                    out[pos] = rec;
                }
                ++pos;
            }
        }
    }
}

template <typename T>
cudaError_t peaks_ctx(const pfc_ctx* c, const void* psi, double ths, void* out, int capacity, cudaStream_t st) {
    const bool d3 = c->nz > 1;
    const int wpr = (c->nx + 31) / 32;
    const int64_t nwords = (int64_t)c->nz * c->ny * wpr;
    const int nchunks = (int)((nwords + kChunkWords - 1) / kChunkWords);
    dim3 grid(wpr, (c->ny + kTY - 1) / kTY, d3 ? (c->nz + kZC - 1) / kZC : 1);
    if (std::is_same<T, float>::value && d3 && c->nx % 128 == 0 && c->ny % kRows4 == 0 &&
        ((uintptr_t)psi & 15) == 0)
        k_peaks_mark4<<<dim3(c->nx / 128, c->ny / kRows4, (c->nz + kZC4 - 1) / kZC4), 32 * (kRows4 + 2),
                        kMark4Smem, st>>>((const float*)psi, c->nx, c->ny, c->nz, (float)ths, c->peak_mask,
                                                 wpr);
    else if (d3)
        k_peaks_mark<T, true><<<grid, dim3(kTX, kTY), 0, st>>>((const T*)psi, c->nx, c->ny, c->nz, (T)ths,
                                                                       c->peak_mask, wpr);
    else
        k_peaks_mark<T, false><<<grid, dim3(kTX, kTY), 0, st>>>((const T*)psi, c->nx, c->ny, c->nz, (T)ths,
                                                                        c->peak_mask, wpr);
    k_words_count<<<nchunks, 256, 0, st>>>(c->peak_mask, nwords, c->peak_counts);
    k_scan<<<1, 1024, 0, st>>>(c->peak_counts, nchunks, c->peak_offsets);
    if (capacity > 0 && out)
        k_peaks_emit<T><<<nchunks, 256, 0, st>>>((const T*)psi, c->peak_mask, nwords, c->nx, c->ny, wpr,
                                                        c->peak_offsets, (MaxRec<T>*)out, capacity);
    return cudaGetLastError();
}

}  // namespace

cudaError_t set_peak_attributes() {
    return cudaFuncSetAttribute(k_peaks_mark4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMark4Smem);
}

int64_t peak_mask_words(int nx, int ny, int nz) { return (int64_t)nz * ny * ((nx + 31) / 32); }
int peak_chunks(int nx, int ny, int nz) {
    return (int)((peak_mask_words(nx, ny, nz) + kChunkWords - 1) / kChunkWords);
}

cudaError_t launch_findpeaks(const pfc_ctx* c, const void* psi, double ths, void* out, int capacity,
                             cudaStream_t st) {
    return c->dtype == PFC_F64 ? peaks_ctx<double>(c, psi, ths, out, capacity, st)
                               : peaks_ctx<float>(c, psi, ths, out, capacity, st);
}

}  // namespace pfc

// ---------------------------------------------------------------------------------------
// Peak finding that allocates nothing.  Its scratch -- the per-block counts of the
// compaction and their scan -- lives in this file-scope device array, sized for grids of
// at most kStaticPeakCells cells (512^3); every GPU that loads the library holds it
// (4 MiB) until the process exits.  Host code must not pass the array's name to a
// kernel: on the host it is only a stand-in for the symbol.  The device address is
// looked up by the first call on a device, with that device current
// (cudaGetSymbolAddress), and cached per device and primary context: a call after
// cudaDeviceReset (a new context, in which the module and its array are loaded afresh)
// looks it up again.
// ---------------------------------------------------------------------------------------
namespace {
constexpr int64_t kStaticPeakCells = (int64_t)1 << 27;
constexpr int kStaticPeakBlocks = (int)(kStaticPeakCells / pfc::kPeakBlock);
static __device__ __align__(256) int g_peak_scratch[2 * kStaticPeakBlocks + 1];
constexpr int kMaxDevices = 64;
struct StaticScratch {
    CUcontext ctx;  // the context the address belongs to
    int* ptr;
};
StaticScratch g_peak_scratch_dev[kMaxDevices];
std::mutex g_peak_scratch_mutex;

// The current context of the calling thread, through the driver entry point that the
// runtime hands out (no link-time dependency on the driver library).
CUcontext current_context() {
    using GetCurrent = CUresult (*)(CUcontext*);
    static GetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (GetCurrent)p;
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}
}  // namespace

extern "C" pfc_status pfc_findpeaks_static(const void* psi, int nx, int ny, int nz, int dtype, double ths,
                                           void* out_maxima, int capacity, int* n_found, void* cuda_stream) {
    if (!psi || !n_found || nx < 1 || ny < 1 || nz < 1 || capacity < 0 || (capacity > 0 && !out_maxima) ||
        (dtype != PFC_F32 && dtype != PFC_F64) || (nz == 1 && !(nx > 1 && ny > 1)))
        return PFC_ERR_INVALID;
    const int64_t cells = (int64_t)nx * ny * nz;
    if (cells > kStaticPeakCells) {
        fprintf(stderr, "pfc_findpeaks_static: %lld cells exceed the static scratch maximum of %lld cells (512^3)\n",
                (long long)cells, (long long)kStaticPeakCells);
        return PFC_ERR_CAPACITY;
    }
    // an error left pending by earlier work of the caller is reported as such, not
    // taken for (and cleared as) a failure of this call's launches
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        fprintf(stderr, "pfc_findpeaks_static: a CUDA error was pending before the call: %s\n",
                cudaGetErrorString(pending));
        return PFC_ERR_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PFC_ERR_CUDA;
    int* scratch;
    {
        std::lock_guard<std::mutex> lock(g_peak_scratch_mutex);
        // cudaFree(0) makes the device's primary context current (the runtime API's
        // initialisation of the device); the driver's current context then names it
        if (cudaFree(0) != cudaSuccess) return PFC_ERR_CUDA;
        const CUcontext cur = current_context();
        if (!cur) return PFC_ERR_CUDA;
        StaticScratch& slot = g_peak_scratch_dev[dev];
        if (!slot.ptr || slot.ctx != cur) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_peak_scratch) != cudaSuccess || !p) return PFC_ERR_CUDA;
            slot.ptr = (int*)p;
            slot.ctx = cur;
        }
        scratch = slot.ptr;
    }
    // counts and offsets are rewritten in full by every call: nothing needs clearing
    int* counts = scratch;
    int* offsets = scratch + kStaticPeakBlocks;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    cudaError_t e = dtype == PFC_F64
                        ? pfc::peaks_raw<double>(psi, nx, ny, nz, ths, counts, offsets, out_maxima, capacity, st)
                        : pfc::peaks_raw<float>(psi, nx, ny, nz, ths, counts, offsets, out_maxima, capacity, st);
    if (e != cudaSuccess) return PFC_ERR_CUDA;
    const int nb = (int)((cells + pfc::kPeakBlock - 1) / pfc::kPeakBlock);
    int total = 0;
    if (cudaMemcpyAsync(&total, offsets + nb, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PFC_ERR_CUDA;
    *n_found = total;
    return total > capacity ? PFC_ERR_CAPACITY : PFC_OK;
}
