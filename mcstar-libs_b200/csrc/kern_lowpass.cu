// The reference's spectral low-pass post-processing of 2D fields, as mirror kernels of its
// arithmetic and its text dump:
//
//  k_gaussian_init   g_k = (e, 1 - e), e = exp(-1/2 sum_a (1.1 d h_a K_a)^2)
//                    (cuda/kernels/gaussian.hpp:23-39; exp in the field's precision)
//  k_kmult           a_k *= Re g_k or Im g_k (gaussian.hpp:41-67, lowpass.hpp:1-35)
//  k_norm_square     psi <- (psi / N)^2, the reference's norm then square
//                    (cuda/kernels/norm.hpp:1-10, lowpass.hpp:37-52) in one sweep
//  write_lowpass     the LOWPASS dump of a low-passed spectrum (lowpass.hpp:54-77): a
//                    header line, the length of a protocol-0 pickle of {n0, n1, l0, l1},
//                    that pickle, then "i0 i1 re im" per mode with |a_k|^2 > 1e-6 (i0 outer,
//                    iostream's default %g formatting), gzip-compressed.  The text is the
//                    reference's byte for byte.  It is formatted by all host threads over
//                    contiguous i0 ranges and compressed as independent 1 MB deflate chunks
//                    (the reference's level; each primed with the previous 32 KB, joined by
//                    sync flushes, one gzip member with the combined CRC-32, as pigz does):
//                    the same decompressed bytes; an output of one chunk is also the same
//                    file as zlib's gzwrite writes.
#include <zlib.h>
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "pfc_ctx.h"

namespace pfc {
namespace {

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    const size_t cap = 148 * 16;
    return (int)(g < cap ? (g ? g : 1) : cap);
}

__device__ __forceinline__ float t_exp(float x) { return expf(x); }
__device__ __forceinline__ double t_exp(double x) { return exp(x); }

template <typename T>
__global__ void k_gaussian_init(cx<T>* g, int nx, int ny, int nz, T lx, T ly, T lz, T hx, T hy, T hz, T dps) {
    const int nxh = nx / 2 + 1;
    const int64_t n = (int64_t)nxh * ny * nz;
    const T sx = T(1.1) * dps * hx, sy = T(1.1) * dps * hy, sz = T(1.1) * dps * hz;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(idx % nxh);
        const int64_t r = idx / nxh;
        const int i1 = (int)(r % ny), i2 = (int)(r / ny);
        const T a = sx * kwave<T>(i0, nx, lx), b = sy * kwave<T>(i1, ny, ly), c = sz * kwave<T>(i2, nz, lz);
        const T e = t_exp(-T(0.5) * (a * a + b * b + c * c));
        g[idx] = cx<T>{e, T(1) - e};
    }
}

template <typename T, bool kImag>
__global__ void k_kmult(cx<T>* a, const cx<T>* __restrict__ g, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const cx<T> v = a[i];
        const T s = kImag ? g[i].y : g[i].x;
        a[i] = cx<T>{s * v.x, s * v.y};
    }
}

template <typename T, bool kNorm>
__global__ void k_norm_square(T* __restrict__ a, int64_t n, T nf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T v = kNorm ? a[i] / nf : a[i];
        a[i] = v * v;
    }
}

int host_threads(int cap) {
    const int n = (int)std::thread::hardware_concurrency();
    return std::max(1, std::min(n > 0 ? n : 1, cap));
}

// Runs f(i) for i < n on up to nt threads (dynamic assignment).
template <class F>
void parallel_for(int n, int nt, F f) {
    std::atomic<int> next{0};
    auto work = [&] {
        for (int i = next++; i < n; i = next++) f(i);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < std::min(nt, n); ++t) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
}

template <typename T>
std::string lowpass_text(const cx<T>* h, int nx, int ny, double lx, double ly) {
    const int nxh = nx / 2 + 1;
    char pickle[256], head[32];
    std::snprintf(pickle, sizeof pickle, "(S'n0'\nI%d\nS'n1'\nI%d\nS'l0'\nF%f\nS'l1'\nF%f\nd.\n", nx, ny, (double)(T)lx,
                  (double)(T)ly);
    std::snprintf(head, sizeof head, "LOWPASS\n%d\n", (int)std::strlen(pickle));
    const int nparts = std::min(nxh, 4 * host_threads(64));
    std::vector<std::string> part(nparts);
    parallel_for(nparts, host_threads(64), [&](int p) {
        char line[96];
        std::string& s = part[p];
        for (int i0 = (int)((int64_t)p * nxh / nparts); i0 < (int)((int64_t)(p + 1) * nxh / nparts); ++i0)
            for (int i1 = 0; i1 < ny; ++i1) {
                const cx<T> v = h[(size_t)i1 * nxh + i0];
                const T m = v.x * v.x + v.y * v.y;
                if (m > 1e-6) {
                    const int k = std::snprintf(line, sizeof line, "%d %d %g %g\n", i0, i1, (double)v.x, (double)v.y);
                    s.append(line, (size_t)k);
                }
            }
    });
    size_t total = std::strlen(head) + std::strlen(pickle);
    for (auto& p : part) total += p.size();
    std::string s;
    s.reserve(total);
    s.append(head).append(pickle);
    for (auto& p : part) s.append(p);
    return s;
}

// gzip file of s: 10-byte header (no name, mtime 0, OS 3, as zlib's gzopen "wb"), the
// deflate chunks, CRC-32 and length.  false when a zlib call or the file write fails.
bool write_gzip(const std::string& s, const char* path) {
    constexpr size_t kChunk = 1 << 20, kDict = 32768;
    const size_t n = s.size();
    const int nch = (int)std::max<size_t>(1, (n + kChunk - 1) / kChunk);
    std::vector<std::string> out(nch);
    std::vector<uLong> crc(nch);
    std::atomic<bool> ok{true};
    parallel_for(nch, host_threads(64), [&](int i) {
        const size_t a = (size_t)i * kChunk, len = std::min(kChunk, n - std::min(n, a));
        z_stream z{};
        if (deflateInit2(&z, Z_DEFAULT_COMPRESSION, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY) != Z_OK) {
            ok = false;
            return;
        }
        if (i > 0) {
            const size_t d = std::min(kDict, a);
            deflateSetDictionary(&z, (const Bytef*)s.data() + a - d, (uInt)d);
        }
        std::string& o = out[i];
        o.resize(deflateBound(&z, (uLong)len) + 64);
        z.next_in = (Bytef*)s.data() + a;
        z.avail_in = (uInt)len;
        z.next_out = (Bytef*)&o[0];
        z.avail_out = (uInt)o.size();
        const int r = deflate(&z, i == nch - 1 ? Z_FINISH : Z_SYNC_FLUSH);
        if (r != (i == nch - 1 ? Z_STREAM_END : Z_OK) || z.avail_in != 0) ok = false;
        o.resize(o.size() - z.avail_out);
        deflateEnd(&z);
        crc[i] = crc32(0L, (const Bytef*)s.data() + a, (uInt)len);
    });
    if (!ok) return false;
    uLong c = crc[0];
    for (int i = 1; i < nch; ++i) c = crc32_combine(c, crc[i], (z_off_t)std::min(kChunk, n - (size_t)i * kChunk));
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    const unsigned char head[10] = {0x1f, 0x8b, 8, 0, 0, 0, 0, 0, 0, 3};
    bool w = std::fwrite(head, 1, 10, f) == 10;
    for (auto& o : out) w = w && std::fwrite(o.data(), 1, o.size(), f) == o.size();
    unsigned char tail[8];
    const uint32_t isz = (uint32_t)n;
    for (int b = 0; b < 4; ++b) {
        tail[b] = (unsigned char)((c >> (8 * b)) & 0xff);
        tail[4 + b] = (unsigned char)((isz >> (8 * b)) & 0xff);
    }
    w = w && std::fwrite(tail, 1, 8, f) == 8;
    return std::fclose(f) == 0 && w;
}

}  // namespace

cudaError_t launch_gaussian_init(const pfc_ctx* c, void* g, double lx, double ly, double lz, double hx, double hy,
                                 double hz, double dps) {
    const int gs = grid_for(c->n_cmpl, 256);
    if (c->dtype == PFC_F64)
        k_gaussian_init<double><<<gs, 256, 0, c->stream>>>((cx<double>*)g, c->nx, c->ny, c->nz, lx, ly, lz, hx, hy, hz,
                                                           dps);
    else
        k_gaussian_init<float><<<gs, 256, 0, c->stream>>>((cx<float>*)g, c->nx, c->ny, c->nz, (float)lx, (float)ly,
                                                          (float)lz, (float)hx, (float)hy, (float)hz, (float)dps);
    return cudaGetLastError();
}

cudaError_t launch_kmult(const pfc_ctx* c, void* a, const void* g, int imag) {
    const int64_t n = (int64_t)c->n_cmpl;
    const int gs = grid_for(c->n_cmpl, 256);
    if (c->dtype == PFC_F64) {
        if (imag) k_kmult<double, true><<<gs, 256, 0, c->stream>>>((cx<double>*)a, (const cx<double>*)g, n);
        else k_kmult<double, false><<<gs, 256, 0, c->stream>>>((cx<double>*)a, (const cx<double>*)g, n);
    } else {
        if (imag) k_kmult<float, true><<<gs, 256, 0, c->stream>>>((cx<float>*)a, (const cx<float>*)g, n);
        else k_kmult<float, false><<<gs, 256, 0, c->stream>>>((cx<float>*)a, (const cx<float>*)g, n);
    }
    return cudaGetLastError();
}

cudaError_t launch_norm_square(const pfc_ctx* c, void* a, int norm) {
    const int64_t n = (int64_t)c->n_real;
    const int gs = grid_for(c->n_real, 256);
    if (c->dtype == PFC_F64) {
        if (norm) k_norm_square<double, true><<<gs, 256, 0, c->stream>>>((double*)a, n, (double)n);
        else k_norm_square<double, false><<<gs, 256, 0, c->stream>>>((double*)a, n, (double)n);
    } else {
        if (norm) k_norm_square<float, true><<<gs, 256, 0, c->stream>>>((float*)a, n, (float)n);
        else k_norm_square<float, false><<<gs, 256, 0, c->stream>>>((float*)a, n, (float)n);
    }
    return cudaGetLastError();
}

// The LOWPASS dump of the device spectrum (already multiplied by the low-pass): copied to
// the host on the context's stream, formatted, written with one gzwrite.  Returns 0, 1 when
// a CUDA call failed (cuda_err set), 2 when the file could not be written.
int write_lowpass_file(const pfc_ctx* c, const void* spectrum, double lx, double ly, const char* path,
                       cudaError_t* cuda_err) {
    std::vector<unsigned char> h(c->state_bytes);
    cudaError_t e = cudaMemcpyAsync(h.data(), spectrum, c->state_bytes, cudaMemcpyDeviceToHost, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    if (e) {
        *cuda_err = e;
        return 1;
    }
    const std::string s = c->dtype == PFC_F64
                              ? lowpass_text<double>((const cx<double>*)h.data(), c->nx, c->ny, lx, ly)
                              : lowpass_text<float>((const cx<float>*)h.data(), c->nx, c->ny, lx, ly);
    return write_gzip(s, path) ? 0 : 2;
}

}  // namespace pfc
