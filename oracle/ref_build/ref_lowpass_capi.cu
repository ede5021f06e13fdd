/* ORACLE / TEST INFRASTRUCTURE ONLY -- never part of the product path.
 *
 * A driver translation unit for the reference's spectral low-pass headers
 * (cuda/kernels/gaussian.hpp, cuda/kernels/lowpass.hpp with common/zstream.hpp and
 * cuda/kernels/norm.hpp), in the pattern of cufft_unittest/main.cu:6-16: it typedefs the
 * reference's Float/GPUArray/... and exposes, through extern "C" functions with host
 * buffers, its Gaussian filter (call_kernel_gaussian_init), its LOWPASS writer
 * (write_lowpass_2d) and its amplitude chain (calc_amplitude_lowpass), so that tests can
 * run the unmodified reference on a B200.  Compiled once per precision (-DFLOAT=float /
 * double) with compat_cuda12.h force-included.  See oracle/Makefile.
 */
#include <chrono>
#include <iostream>
#include <sstream>
#include <string>
#include <common/zstream.hpp>
#include <cuda/array_abstraction.hpp>
#include <cuda/cufft_wrapper.hpp>

typedef FLOAT Float;
typedef Array::TP<Float>::CT Float2;
#if defined(REF_F64)
typedef double3 Float3;
#define REFL(name) refl64_##name
#else
typedef float3 Float3;
#define REFL(name) refl32_##name
#endif
typedef Array::CPUArray<Float> CPUArray;
typedef Array::GPUArray<Float> GPUArray;
typedef FFT::CufftPlan<Float, FFT::R2C> PlanR2C;
typedef FFT::CufftPlan<Float, FFT::C2R> PlanC2R;

#include <cuda/kernels/gaussian.hpp>  // includes cuda/kernels/common.hpp, which norm.hpp needs
#include <cuda/kernels/norm.hpp>
#include <cuda/kernels/lowpass.hpp>

namespace {
Float3 mk3(double x, double y, double z) { Float3 r; r.x = Float(x); r.y = Float(y); r.z = Float(z); return r; }
size_t cmpl_bytes(int3 s) { return (size_t)(s.x / 2 + 1) * s.y * s.z * sizeof(Float2); }
}

extern "C" {

/* kgauss (half spectrum, host) of call_kernel_gaussian_init */
void REFL(gaussian_init)(int nx, int ny, int nz, double lx, double ly, double lz, double hx, double hy, double hz,
                         double dps, void* kgauss_out) {
    const int3 shape{nx, ny, nz};
    CPUArray host(shape);
    GPUArray g(shape);
    call_kernel_gaussian_init(g, mk3(lx, ly, lz), mk3(hx, hy, hz), Float(dps));
    g >> host;
    std::memcpy(kgauss_out, host.ptr_void(), cmpl_bytes(shape));
}

/* write_lowpass_2d of a host spectrum and filter (2D) */
void REFL(write_lowpass_2d)(int nx, int ny, const void* spectrum_in, const void* kgauss_in, double lx, double ly,
                            const char* fn) {
    const int3 shape{nx, ny, 1};
    CPUArray host(shape);
    GPUArray spec(shape), g(shape);
    std::memcpy(host.ptr_void(), spectrum_in, cmpl_bytes(shape));
    host >> spec;
    std::memcpy(host.ptr_void(), kgauss_in, cmpl_bytes(shape));
    host >> g;
    write_lowpass_2d(spec, g, host, mk3(lx, ly, 1.0), std::string(fn));
}

/* calc_amplitude_lowpass of a host spectrum and filter (2D): the amplitude field (real,
 * nx ny values) into amp_out, the LOWPASS dump to fn */
void REFL(amplitude_lowpass)(int nx, int ny, const void* spectrum_in, const void* kgauss_in, double lx, double ly,
                             const char* fn, void* amp_out) {
    const int3 shape{nx, ny, 1};
    CPUArray host(shape);
    GPUArray spec(shape), aux(shape), g(shape);
    PlanR2C r2c(shape);
    PlanC2R c2r(shape);
    std::memcpy(host.ptr_void(), spectrum_in, cmpl_bytes(shape));
    host >> spec;
    std::memcpy(host.ptr_void(), kgauss_in, cmpl_bytes(shape));
    host >> g;
    calc_amplitude_lowpass(r2c, c2r, spec, aux, g, host, mk3(lx, ly, 1.0), std::string(fn));
    std::memcpy(amp_out, host.ptr_real(), (size_t)nx * ny * sizeof(Float));
}

/* timing of calc_amplitude_lowpass with the arrays and plans made once: each of `calls`
 * iterations restores the spectrum (device copy) and runs the chain, dump to fn included;
 * returns the elapsed milliseconds (host clock around device-synchronised calls) */
double REFL(time_amplitude_lowpass)(int nx, int ny, const void* spectrum_in, const void* kgauss_in, double lx,
                                    double ly, const char* fn, int warmup, int calls) {
    const int3 shape{nx, ny, 1};
    CPUArray host(shape);
    GPUArray spec0(shape), spec(shape), aux(shape), g(shape);
    PlanR2C r2c(shape);
    PlanC2R c2r(shape);
    std::memcpy(host.ptr_void(), spectrum_in, cmpl_bytes(shape));
    host >> spec0;
    std::memcpy(host.ptr_void(), kgauss_in, cmpl_bytes(shape));
    host >> g;
    for (int i = 0; i < warmup; ++i) {
        spec0 >> spec;
        calc_amplitude_lowpass(r2c, c2r, spec, aux, g, host, mk3(lx, ly, 1.0), std::string(fn));
    }
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < calls; ++i) {
        spec0 >> spec;
        calc_amplitude_lowpass(r2c, c2r, spec, aux, g, host, mk3(lx, ly, 1.0), std::string(fn));
    }
    cudaDeviceSynchronize();
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
