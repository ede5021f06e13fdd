// Local-maximum peak finding (cuda/kernels/findpeaks.hpp:7-29, findpeaks_2d.hpp:7-27).
// A cell is a peak when it is strictly greater than all 26 (3D) or 8 (2D) periodic
// neighbours and >= ths.  Deterministic compaction: pass 1 counts peaks per block of
// kPeakBlock consecutive cells (__syncthreads_count), one block scans the counts,
// pass 2 writes each peak at block offset + warp-ballot rank.  Blocks cover linear
// index ranges in order, so the output is sorted by linear index.
#include <cuda.h>
#include <cstdio>
#include <mutex>
#include "pfc_ctx.h"

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

}  // namespace

cudaError_t launch_findpeaks(const pfc_ctx* c, const void* psi, double ths, void* out, int capacity) {
    return c->dtype == PFC_F64
               ? peaks_raw<double>(psi, c->nx, c->ny, c->nz, ths, c->peak_counts, c->peak_offsets, out, capacity,
                                   c->stream)
               : peaks_raw<float>(psi, c->nx, c->ny, c->nz, ths, c->peak_counts, c->peak_offsets, out, capacity,
                                  c->stream);
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
