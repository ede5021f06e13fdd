// Plumbing shared by the mcstar-libs-named headers in this directory, which forward
// the reference's source-level API to the C ABI of libpfc_b200 (include/pfc_b200.h).
//
//  * One pfc_ctx per (grid shape, precision), created on first use and kept for the
//    life of the process (the reference's call_kernel_* functions take only arrays).
//  * Every non-zero pfc_status is printed with the context's message and ends the
//    process, which is what the reference's CUERR/CUFFTERR/CURAND_CALL do
//    (common/cu_error.hpp:5-11, cuda/cufft_wrapper.hpp:30-38, cuda/curand_error.hpp:4).
//  * Every forwarded call synchronises the device afterwards, as the reference's
//    wrappers do with cudaThreadSynchronize, so host code that reads results right
//    after a call keeps working.
//  * A minimal .npy (format 1.0) reader and writer for CPUArray::load / save.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../pfc_b200.h"

namespace pfc_shim {

inline void check(pfc_status s, const pfc_ctx* c, const char* what, const char* file, int line) {
    if (s == PFC_OK) return;
    fprintf(stderr, "PFCERR: %s: %s (%s) %s:%d\n", what, pfc_status_string(s), c ? pfc_last_error(c) : "", file,
            line);
    fflush(stderr);
    exit(EXIT_FAILURE);
}

inline void sync(const char* file, int line) {
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        fprintf(stderr, "CUERR: %s %s:%d\n", cudaGetErrorString(e), file, line);
        fflush(stderr);
        exit(EXIT_FAILURE);
    }
}

template <typename F> struct dtype_of;
template <> struct dtype_of<float> { static constexpr int value = PFC_F32; };
template <> struct dtype_of<double> { static constexpr int value = PFC_F64; };

// The context of grids of this shape (x fastest) and precision.
template <typename F>
inline pfc_ctx* context(int3 shape) {
    static std::map<std::tuple<int, int, int>, pfc_ctx*> cache;
    const auto key = std::make_tuple(shape.x, shape.y, shape.z);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    pfc_desc d;
    d.nx = shape.x;
    d.ny = shape.y;
    d.nz = shape.z;
    d.dtype = dtype_of<F>::value;
    pfc_ctx* c = nullptr;
    check(pfc_create(&d, &c), nullptr, "pfc_create", __FILE__, __LINE__);
    cache.emplace(key, c);
    return c;
}

// ---- .npy format 1.0: magic, version, little-endian header length, a Python dict
// literal padded with spaces to a multiple of 64 bytes, then the raw C-order data ----
template <typename T> struct npy_descr;
template <> struct npy_descr<float> { static const char* get() { return "<f4"; } };
template <> struct npy_descr<double> { static const char* get() { return "<f8"; } };
template <> struct npy_descr<float2> { static const char* get() { return "<c8"; } };
template <> struct npy_descr<double2> { static const char* get() { return "<c16"; } };

// shape: numpy order (slowest first), `dims` entries
template <typename T>
inline void npy_save(const std::string& fn, int dims, const int* shape, const void* data) {
    std::string dict = std::string("{'descr': '") + npy_descr<T>::get() + "', 'fortran_order': False, 'shape': (";
    size_t count = 1;
    for (int i = 0; i < dims; ++i) {
        dict += std::to_string(shape[i]) + (dims == 1 ? ",)" : (i + 1 < dims ? ", " : ")"));
        count *= (size_t)shape[i];
    }
    dict += ", }";
    const size_t pre = 10;  // magic (6) + version (2) + header length (2)
    size_t total = pre + dict.size() + 1;
    const size_t pad = (64 - total % 64) % 64;
    dict += std::string(pad, ' ') + "\n";
    FILE* f = fopen(fn.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + fn + " for writing");
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const uint16_t hl = (uint16_t)dict.size();
    const unsigned char hlb[2] = {(unsigned char)(hl & 0xff), (unsigned char)(hl >> 8)};
    bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(hlb, 1, 2, f) == 2 &&
              fwrite(dict.data(), 1, dict.size(), f) == dict.size() &&
              fwrite(data, sizeof(T), count, f) == count;
    fclose(f);
    if (!ok) throw std::runtime_error("short write to " + fn);
}

// Reads a C-order array of element type T; returns its shape (slowest first).
template <typename T>
inline std::vector<int> npy_load(const std::string& fn, std::vector<T>& data) {
    FILE* f = fopen(fn.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + fn);
    unsigned char head[10];
    if (fread(head, 1, 10, f) != 10 || head[0] != 0x93 || memcmp(head + 1, "NUMPY", 5) != 0) {
        fclose(f);
        throw std::runtime_error(fn + ": not a .npy file");
    }
    size_t hl = head[8] | ((size_t)head[9] << 8);
    if (head[6] >= 2) {  // format 2.0/3.0: four-byte header length
        unsigned char more[2];
        if (fread(more, 1, 2, f) != 2) { fclose(f); throw std::runtime_error(fn + ": truncated"); }
        hl |= ((size_t)more[0] << 16) | ((size_t)more[1] << 24);
    }
    std::string dict(hl, ' ');
    if (fread(&dict[0], 1, hl, f) != hl) { fclose(f); throw std::runtime_error(fn + ": truncated header"); }
    if (dict.find(npy_descr<T>::get()) == std::string::npos || dict.find("'fortran_order': False") == std::string::npos) {
        fclose(f);
        throw std::runtime_error(fn + ": element type or order differs from the array's");
    }
    std::vector<int> shape;
    const size_t a = dict.find('(', dict.find("'shape'")), b = dict.find(')', a);
    std::string s = dict.substr(a + 1, b - a - 1);
    size_t count = 1, p = 0;
    while (p < s.size()) {
        while (p < s.size() && (s[p] == ' ' || s[p] == ',')) ++p;
        if (p >= s.size()) break;
        const int v = atoi(s.c_str() + p);
        shape.push_back(v);
        count *= (size_t)v;
        while (p < s.size() && s[p] != ',') ++p;
    }
    data.resize(count);
    const size_t got = fread(data.data(), sizeof(T), count, f);
    fclose(f);
    if (got != count) throw std::runtime_error(fn + ": truncated data");
    return shape;
}

}  // namespace pfc_shim

#define PFC_SHIM_CHECK(call, ctx) pfc_shim::check((call), (ctx), #call, __FILE__, __LINE__)
#define PFC_SHIM_SYNC() pfc_shim::sync(__FILE__, __LINE__)
