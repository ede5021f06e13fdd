// Array::GPUArray / CPUArray with the interface of mcstar-libs
// cuda/array_abstraction.hpp:14-211, so host code written against it compiles
// unchanged.  A GPUArray owns a cudaMalloc buffer of the half-spectrum size (S bytes,
// enough for the real field too); a CPUArray owns pinned host memory of the same size.
// .npy files are read and written by pfc_shim (format 1.0, C order).
#pragma once
#include <cuda_runtime.h>
#include <sys/mman.h>

#include <cassert>
#include <complex>
#include <cstring>
#include <functional>
#include <future>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../common/cu_error.hpp"
#include "../common/technicalities.hpp"
#include "../pfc_shim.hpp"

namespace Array {

struct AsReal {};
struct AsCmpl {};

// real and complex element types of a precision
template <typename> struct TP {};
template <> struct TP<float> {
    typedef float RT;
    typedef float2 CT;
};
template <> struct TP<double> {
    typedef double RT;
    typedef double2 CT;
};

template <typename F> class Array {
  protected:
    F* m_ptr;
    const int m_dims;
    int m_real_elems;
    int3 m_ext_real;
    int3 m_ext_cmpl;
    int m_cmpl_elems;
    size_t m_bytes;
    explicit Array(int3 ext)
        : m_ptr(nullptr),
          m_dims(ext.z == 1 ? (ext.y == 1 ? 1 : 2) : 3),
          m_real_elems(ext.x * ext.y * ext.z),
          m_ext_real(ext),
          m_ext_cmpl(int3{ext.x / 2 + 1, ext.y, ext.z}),
          m_cmpl_elems((ext.x / 2 + 1) * ext.y * ext.z),
          m_bytes((size_t)(ext.x / 2 + 1) * ext.y * ext.z * 2 * sizeof(F)) {
        if (ext.x < 1 || ext.y < 1 || ext.z < 1) throw std::runtime_error("extent must be >=1 in all dimensions");
    }

  public:
    int real_elems() { return m_real_elems; }
    int cmpl_elems() { return m_cmpl_elems; }
    int3 real_vext() { return m_ext_real; }
    int3 cmpl_vext() { return m_ext_cmpl; }
    int real_ext(int i) { return i == 0 ? m_ext_real.x : (i == 1 ? m_ext_real.y : m_ext_real.z); }
    int cmpl_ext(int i) { return i == 0 ? m_ext_cmpl.x : (i == 1 ? m_ext_cmpl.y : m_ext_cmpl.z); }
    void* ptr_void() { return m_ptr; }
    F* ptr_real() { return m_ptr; }
    typename TP<F>::CT* ptr_cmpl() { return reinterpret_cast<typename TP<F>::CT*>(m_ptr); }

    typedef F RT;
    typedef typename TP<F>::CT CT;
};

template <typename> struct CPUArray;

template <typename F> struct GPUArray : public Array<F> {
    explicit GPUArray(CPUArray<F>& from) : Array<F>(from.real_vext()) {
        CUERR(cudaMalloc((void**)&this->m_ptr, this->m_bytes));
        from >> (*this);
    }
    explicit GPUArray(int3 ext) : Array<F>(ext) { CUERR(cudaMalloc((void**)&this->m_ptr, this->m_bytes)); }
    GPUArray(const GPUArray&) = delete;
    GPUArray& operator=(const GPUArray&) = delete;
    ~GPUArray() { CUERR(cudaFree(this->m_ptr)); }
    void operator>>(GPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        CUERR(cudaMemcpy(o.ptr_void(), this->m_ptr, this->m_bytes, cudaMemcpyDeviceToDevice));
    }
    void operator>>(CPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        CUERR(cudaMemcpy(o.ptr_void(), this->m_ptr, this->m_bytes, cudaMemcpyDeviceToHost));
    }
    // exchange the buffers of two arrays of the same extent
    void operator%(GPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        F* p = o.m_ptr;
        o.m_ptr = this->m_ptr;
        this->m_ptr = p;
    }
};

template <typename F> struct CPUArray : public Array<F> {
    explicit CPUArray(CPUArray<F>& from) : Array<F>(from.real_vext()) {
        alloc();
        from >> (*this);
    }
    explicit CPUArray(int3 ext) : Array<F>(ext) {
        alloc();
        memset(this->m_ptr, 0, this->m_bytes);
    }
    CPUArray(const CPUArray&) = delete;
    CPUArray& operator=(const CPUArray&) = delete;
    ~CPUArray() { CUERR(cudaFreeHost(this->m_ptr)); }
    void operator>>(CPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        memcpy(o.ptr_void(), this->m_ptr, this->m_bytes);
    }
    void operator>>(GPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        CUERR(cudaMemcpy(o.ptr_void(), this->m_ptr, this->m_bytes, cudaMemcpyHostToDevice));
    }
    void operator%(CPUArray<F>& o) {
        assert(o.real_vext() == this->m_ext_real && "array dimensions differ");
        F* p = o.m_ptr;
        o.m_ptr = this->m_ptr;
        this->m_ptr = p;
    }
    // x-fastest linear index, or (i0, i1, i2) = (x, y, z)
    F& operator[](int idx) { return this->m_ptr[idx]; }
    F& operator[](int3 idx) { return this->m_ptr[(idx.z * this->m_ext_real.y + idx.y) * this->m_ext_real.x + idx.x]; }

    // the real field from a .npy file of this array's (numpy-order) shape; a mismatch
    // is reported and aborts, as the reference does
    void load(const std::string fn) {
        std::vector<F> data;
        const std::vector<int> shape = pfc_shim::npy_load<F>(fn, data);
        int3 ext{1, 1, 1};
        if (shape.size() == 1) ext.x = shape[0];
        else if (shape.size() == 2) { ext.x = shape[1]; ext.y = shape[0]; }
        else if (shape.size() == 3) { ext.x = shape[2]; ext.y = shape[1]; ext.z = shape[0]; }
        else throw std::runtime_error(fn + ": arrays of 1 to 3 dimensions only");
        if (!(ext == this->m_ext_real)) {
            fprintf(stderr, "*** array dimension mismatch");
            fflush(stderr);
            abort();
        }
        memcpy(this->m_ptr, data.data(), (size_t)this->m_real_elems * sizeof(F));
        fprintf(stderr, "*** array initialized from file <%s>\n", fn.c_str());
        fflush(stderr);
    }
    // the real field (AsReal) or the half spectrum (AsCmpl) as a .npy file
    template <typename Kind = AsReal> void save(const std::string fn) { save_as(fn, Kind{}); }

    void over(std::function<void(F&)> f) {
        for (int i = 0; i < this->m_real_elems; ++i) f(this->m_ptr[i]);
    }
    void over(std::function<void(typename TP<F>::CT&)> f) {
        for (int i = 0; i < this->m_cmpl_elems; ++i) f(this->ptr_cmpl()[i]);
    }
    void over(std::function<void(F&, int)> f) {
        for (int i = 0; i < this->m_real_elems; ++i) f(this->m_ptr[i], i);
    }
    void over(std::function<void(typename TP<F>::CT&, int)> f) {
        for (int i = 0; i < this->m_cmpl_elems; ++i) f(this->ptr_cmpl()[i], i);
    }
    void square() { over([](F& v) { v *= v; }); }
    void set_to(F val) { over([val](F& v) { v = val; }); }
    void mult(F val) { over([val](F& v) { v *= val; }); }
    void add(F val) { over([val](F& v) { v += val; }); }
    F max() {
        F m = this->m_ptr[0];
        over([&m](F& v) { m = m > v ? m : v; });
        return m;
    }
    F min() {
        F m = this->m_ptr[0];
        over([&m](F& v) { m = m < v ? m : v; });
        return m;
    }

  private:
    void alloc() {
        CUERR(cudaHostAlloc((void**)&this->m_ptr, this->m_bytes, cudaHostAllocDefault));
        if (mlock(this->m_ptr, this->m_bytes) != 0) std::cerr << "*** host memory not pinned" << std::endl;
    }
    void save_as(const std::string& fn, AsReal) {
        const int3 s = shape_tr(this->m_ext_real);
        const int shape[3] = {s.x, s.y, s.z};
        pfc_shim::npy_save<F>(fn, this->m_dims, shape, this->m_ptr);
    }
    void save_as(const std::string& fn, AsCmpl) {
        const int3 s = shape_tr(this->m_ext_real);
        int shape[3] = {s.x, s.y, s.z};
        shape[this->m_dims - 1] = this->m_ext_cmpl.x;  // the x extent (fastest) is halved
        pfc_shim::npy_save<typename TP<F>::CT>(fn, this->m_dims, shape, this->m_ptr);
    }
};

}  // namespace Array
