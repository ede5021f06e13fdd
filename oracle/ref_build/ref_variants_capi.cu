/* ORACLE / TEST INFRASTRUCTURE ONLY -- never part of the product path.
 *
 * A driver translation unit for the reference's other propagators:
 * cuda/kernels/eom-exp.hpp (exponential conserved update), cuda/kernels/el.hpp and
 * cuda/kernels/el-exp.hpp (non-conserved relaxation).  They cannot share a unit with
 * eom.hpp (both define kernel_calc_fen), hence this separate library.  Every function
 * takes host half spectra, runs the reference's own call on the GPU and copies back.
 * Compiled per precision with -DFLOAT=float|double; see oracle/Makefile.
 */
#include <cstring>
#include <iostream>
#include <cuda/array_abstraction.hpp>

typedef FLOAT Float;
typedef Array::TP<Float>::CT Float2;
#if defined(REF_F64)
typedef double3 Float3;
#define REFV(name) refv64_##name
#else
typedef float3 Float3;
#define REFV(name) refv32_##name
#endif
typedef Array::CPUArray<Float> CPUArray;
typedef Array::GPUArray<Float> GPUArray;

#include <cuda/kernels/eom-exp.hpp>
#include <cuda/kernels/el.hpp>
#include <cuda/kernels/el-exp.hpp>

namespace {
Float3 mk3(double x, double y, double z) { Float3 r; r.x = Float(x); r.y = Float(y); r.z = Float(z); return r; }

struct Fields {
    int3 shape;
    CPUArray host;
    GPUArray a, b, c, d;
    explicit Fields(int nx, int ny, int nz)
        : shape{nx, ny, nz}, host(int3{nx, ny, nz}), a(int3{nx, ny, nz}), b(int3{nx, ny, nz}),
          c(int3{nx, ny, nz}), d(int3{nx, ny, nz}) {}
    size_t bytes() { return (size_t)host.cmpl_elems() * sizeof(Float2); }
    void up(GPUArray& g, const void* src) { std::memcpy(host.ptr_void(), src, bytes()); host >> g; }
    void down(GPUArray& g, void* dst) { g >> host; std::memcpy(dst, host.ptr_void(), bytes()); }
};
}  // namespace

extern "C" {

void REFV(init_eom_op)(int nx, int ny, int nz, double dt, double eps, double lx, double ly, double lz, void* kop) {
    Fields f(nx, ny, nz);
    call_kernel_init_eom_op(f.a, Float(dt), Float(eps), mk3(lx, ly, lz));
    f.down(f.a, kop);
}

/* knoise may be NULL; with_fen also returns L^ psi^_old in knoise_out */
void REFV(update_eom_exp)(int nx, int ny, int nz, const void* kop, void* kpsi, const void* knl, const void* knoise,
                          double namp, double dt, double eps, double lx, double ly, double lz, int with_fen,
                          void* knoise_out) {
    Fields f(nx, ny, nz);
    f.up(f.a, kop);
    f.up(f.b, kpsi);
    f.up(f.c, knl);
    if (knoise) f.up(f.d, knoise);
    if (with_fen)
        call_kernel_update_eom_with_fen(f.a, f.b, f.c, f.d, Float(namp), Float(dt), Float(eps), mk3(lx, ly, lz));
    else if (knoise)
        call_kernel_update_eom(f.a, f.b, f.c, f.d, Float(namp), Float(dt), Float(eps), mk3(lx, ly, lz));
    else
        call_kernel_update_eom(f.a, f.b, f.c, Float(namp), Float(dt), Float(eps), mk3(lx, ly, lz));
    f.down(f.b, kpsi);
    if (with_fen && knoise_out) f.down(f.d, knoise_out);
}

float REFV(update_el)(int nx, int ny, int nz, void* kpsi, const void* knl, double dt, double eps, double lx,
                      double ly, double lz) {
    Fields f(nx, ny, nz);
    f.up(f.a, kpsi);
    f.up(f.b, knl);
    const float m = (float)call_kernel_update_el(f.a, f.b, Float(dt), Float(eps), mk3(lx, ly, lz));
    f.down(f.a, kpsi);
    return m;
}

void REFV(init_el_op)(int nx, int ny, int nz, double dt, double eps, double lx, double ly, double lz, void* kop) {
    Fields f(nx, ny, nz);
    call_kernel_init_el_op(f.a, Float(dt), Float(eps), mk3(lx, ly, lz));
    f.down(f.a, kop);
}

float REFV(update_el_exp)(int nx, int ny, int nz, const void* kop, void* kpsi, const void* knl, double dt,
                          double eps, double lx, double ly, double lz) {
    Fields f(nx, ny, nz);
    f.up(f.a, kop);
    f.up(f.b, kpsi);
    f.up(f.c, knl);
    const float m = (float)call_kernel_update_el(f.a, f.b, f.c, Float(dt), Float(eps), mk3(lx, ly, lz));
    f.down(f.b, kpsi);
    return m;
}

}  // extern "C"
