/* ORACLE / TEST INFRASTRUCTURE ONLY -- never part of the product path.
 *
 * A driver translation unit for the reference's own CUDA headers (the reference
 * ships no main(); its drivers typedef Float/GPUArray/... and include the headers,
 * cufft_unittest/main.cu:6-16 shows the pattern).  It exposes the reference's
 * stock conserved step (cuda/kernels/eom.hpp:60-86, cuda/kernels/psi3_split.hpp,
 * cuda/cufft_wrapper.hpp), its free-energy path (eom.hpp:88-141, norm.hpp), its
 * k-space noise (cuda/noise.hpp:93-150) and its peak finder (findpeaks.hpp,
 * findpeaks_2d.hpp) through extern "C" functions with host buffers, so tests and
 * the reference arm of bench.py can run the unmodified reference on a B200.
 *
 * Compiled once per precision with -DFLOAT=float or -DFLOAT=double (the
 * reference selects precision with that macro, cuda/kernels/common.hpp:16) and
 * with compat_cuda12.h force-included.  See oracle/Makefile.
 */
#include <iostream>
#include <string>
#include <cuda/array_abstraction.hpp>
#include <cuda/cufft_wrapper.hpp>

typedef FLOAT Float;
typedef Array::TP<Float>::CT Float2;
#if defined(REF_F64)
typedef double3 Float3;
#define REFP(name) ref64_##name
#else
typedef float3 Float3;
#define REFP(name) ref32_##name
#endif
typedef Array::CPUArray<Float> CPUArray;
typedef Array::GPUArray<Float> GPUArray;
typedef FFT::CufftPlan<Float, FFT::R2C> PlanR2C;
typedef FFT::CufftPlan<Float, FFT::C2R> PlanC2R;

#include <cuda/noise.hpp>
#include <cuda/kernels/eom.hpp>
#include <cuda/kernels/psi3_split.hpp>
#include <cuda/kernels/norm.hpp>
#include <cuda/kernels/findpeaks.hpp>
#include <cuda/kernels/findpeaks_2d.hpp>

namespace {
struct RefState {
    int3 shape;
    CPUArray* host;
    GPUArray *kpsi, *ktmp, *psi, *knl, *knoise, *lpsi;
    PlanR2C* r2c;
    PlanC2R* c2r;
    NoiseHostApi<Float>* noise;
};
Float3 mk3(double x, double y, double z) { Float3 r; r.x = Float(x); r.y = Float(y); r.z = Float(z); return r; }
}

extern "C" {

void* REFP(create)(int nx, int ny, int nz, unsigned long long seed) {
    RefState* s = new RefState;
    s->shape = int3{nx, ny, nz};
    s->host = new CPUArray(s->shape);
    s->kpsi = new GPUArray(s->shape);
    s->ktmp = new GPUArray(s->shape);
    s->psi = new GPUArray(s->shape);
    s->knl = new GPUArray(s->shape);
    s->knoise = new GPUArray(s->shape);
    s->lpsi = new GPUArray(s->shape);
    s->r2c = new PlanR2C(s->shape);
    s->c2r = new PlanC2R(s->shape);
    s->noise = new NoiseHostApi<Float>(seed);
    return s;
}

void REFP(destroy)(void* h) {
    RefState* s = (RefState*)h;
    delete s->noise; delete s->c2r; delete s->r2c;
    delete s->lpsi; delete s->knoise; delete s->knl; delete s->psi; delete s->ktmp; delete s->kpsi;
    delete s->host;
    delete s;
}

size_t REFP(state_bytes)(void* h) {
    RefState* s = (RefState*)h;
    return (size_t)s->host->cmpl_elems() * 2 * sizeof(Float);
}

/* complex half-spectrum in/out of the state kpsi (host buffer, reference layout) */
void REFP(set_kpsi)(void* h, const void* src) {
    RefState* s = (RefState*)h;
    std::memcpy(s->host->ptr_void(), src, REFP(state_bytes)(h));
    (*s->host) >> (*s->kpsi);
}
void REFP(get_kpsi)(void* h, void* dst) {
    RefState* s = (RefState*)h;
    (*s->kpsi) >> (*s->host);
    std::memcpy(dst, s->host->ptr_void(), REFP(state_bytes)(h));
}

/* unnormalised R2C / C2R through the reference's cuFFT wrapper */
void REFP(r2c)(void* h, const void* real_in, void* cmpl_out) {
    RefState* s = (RefState*)h;
    std::memcpy(s->host->ptr_void(), real_in, (size_t)s->host->real_elems() * sizeof(Float));
    (*s->host) >> (*s->psi);
    s->r2c->execute(*s->psi, *s->ktmp);
    (*s->ktmp) >> (*s->host);
    std::memcpy(cmpl_out, s->host->ptr_void(), REFP(state_bytes)(h));
}
void REFP(c2r)(void* h, const void* cmpl_in, void* real_out) {
    RefState* s = (RefState*)h;
    std::memcpy(s->host->ptr_void(), cmpl_in, REFP(state_bytes)(h));
    (*s->host) >> (*s->ktmp);
    s->c2r->execute(*s->ktmp, *s->psi);
    (*s->psi) >> (*s->host);
    std::memcpy(real_out, s->host->ptr_void(), (size_t)s->host->real_elems() * sizeof(Float));
}

/* The stock conserved step, S times: copy, C2R, psi3_split(norm), R2C,
 * [fill_kspace], update_eom -- the loop every reference driver runs. */
void REFP(step)(void* h, int nsteps, double namp, double dt, double eps,
                double lx, double ly, double lz, double mu, int use_noise) {
    RefState* s = (RefState*)h;
    Float3 lens = mk3(lx, ly, lz);
    for (int t = 0; t < nsteps; ++t) {
        (*s->kpsi) >> (*s->ktmp);
        s->c2r->execute(*s->ktmp, *s->psi);
        call_kernel_psi3_split(*s->psi, NULL, Float(mu), true);
        s->r2c->execute(*s->psi, *s->knl);
        if (use_noise) {
            s->noise->fill_kspace(*s->knoise);
            call_kernel_update_eom(*s->kpsi, *s->knl, *s->knoise, Float(namp), Float(dt), Float(eps), lens);
        } else {
            call_kernel_update_eom(*s->kpsi, *s->knl, Float(namp), Float(dt), Float(eps), lens);
        }
    }
}

/* Device time of nsteps stock steps, CUDA events on the legacy stream. */
float REFP(time_steps)(void* h, int nsteps, double namp, double dt, double eps,
                       double lx, double ly, double lz, double mu, int use_noise) {
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    REFP(step)(h, nsteps, namp, dt, eps, lx, ly, lz, mu, use_noise);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a); cudaEventDestroy(b);
    return ms;
}

/* The pinned host mirror (CPUArray) of the state, for callers that fill it directly. */
void* REFP(host_ptr)(void* h) { return ((RefState*)h)->host->ptr_void(); }

/* End to end: the reference's own pinned H2D (CPUArray >> GPUArray), nsteps stock
 * steps, D2H back (GPUArray >> CPUArray); device time by CUDA events. */
float REFP(time_e2e)(void* h, int nsteps, double namp, double dt, double eps,
                     double lx, double ly, double lz, double mu, int use_noise) {
    RefState* s = (RefState*)h;
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    (*s->host) >> (*s->kpsi);
    REFP(step)(h, nsteps, namp, dt, eps, lx, ly, lz, mu, use_noise);
    (*s->kpsi) >> (*s->host);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a); cudaEventDestroy(b);
    return ms;
}

/* Real field psi = C2R(kpsi)/N into host buffer (reference output path,
 * array_abstraction.hpp + norm.hpp). */
void REFP(get_psi)(void* h, void* real_out) {
    RefState* s = (RefState*)h;
    (*s->kpsi) >> (*s->ktmp);
    s->c2r->execute(*s->ktmp, *s->psi);
    call_kernel_norm(*s->psi);
    (*s->psi) >> (*s->host);
    std::memcpy(real_out, s->host->ptr_void(), (size_t)s->host->real_elems() * sizeof(Float));
}

/* Free energy of the current state via the reference's own path (eom.hpp:88-141):
 * update_eom_with_fen at dt=0 leaves kpsi bit-identical and stores L^psi^ in
 * knoise; then C2R+norm of both and calc_fen.  Returns the float the reference
 * returns; the density is left in lpsi_out (host, real layout) when non-null. */
float REFP(free_energy)(void* h, double eps, double lx, double ly, double lz,
                        double hx, double hy, double hz, void* density_out) {
    RefState* s = (RefState*)h;
    Float3 lens = mk3(lx, ly, lz);
    Float3 hh = mk3(hx, hy, hz);
    cudaMemset(s->knl->ptr_void(), 0, REFP(state_bytes)(h));
    cudaMemset(s->knoise->ptr_void(), 0, REFP(state_bytes)(h));
    call_kernel_update_eom_with_fen(*s->kpsi, *s->knl, *s->knoise, Float(0), Float(0), Float(eps), lens);
    s->c2r->execute(*s->knoise, *s->lpsi);
    call_kernel_norm(*s->lpsi);
    (*s->kpsi) >> (*s->ktmp);
    s->c2r->execute(*s->ktmp, *s->psi);
    call_kernel_norm(*s->psi);
    float f = call_kernel_calc_fen(*s->psi, *s->lpsi, hh);
    if (density_out) {
        (*s->lpsi) >> (*s->host);
        std::memcpy(density_out, s->host->ptr_void(), (size_t)s->host->real_elems() * sizeof(Float));
    }
    return f;
}

/* Peaks (and, in 3D, bond order) of the current real field via the reference's
 * own wrappers, which write their text outputs to the given paths. */
void REFP(findpeaks)(void* h, double hx, double hy, double hz, double lx, double ly, double lz,
                     double ths, double rlim, const char* peaks_fn, const char* bo_fn) {
    RefState* s = (RefState*)h;
    (*s->kpsi) >> (*s->ktmp);
    s->c2r->execute(*s->ktmp, *s->psi);
    call_kernel_norm(*s->psi);
    Float3 hh = mk3(hx, hy, hz), len = mk3(lx, ly, lz);
    if (s->shape.z == 1)
        call_kernel_findpeaks_2d(*s->psi, std::string(peaks_fn), hh, len, Float(ths));
    else
        call_kernel_findpeaks(*s->psi, std::string(peaks_fn), std::string(bo_fn), hh, len, Float(ths), Float(rlim));
}

/* One draw of the reference's k-space noise (noise.hpp:110-142) into host memory. */
void REFP(noise_kspace)(void* h, void* cmpl_out) {
    RefState* s = (RefState*)h;
    s->noise->fill_kspace(*s->knoise);
    (*s->knoise) >> (*s->host);
    std::memcpy(cmpl_out, s->host->ptr_void(), REFP(state_bytes)(h));
}

static void up(RefState* s, GPUArray* a, const void* src, size_t bytes) {
    std::memcpy(s->host->ptr_void(), src, bytes);
    (*s->host) >> (*a);
}
static void down(RefState* s, GPUArray* a, void* dst, size_t bytes) {
    (*a) >> (*s->host);
    std::memcpy(dst, s->host->ptr_void(), bytes);
}

/* The polynomial-kernel update (eom.hpp:143-180) on host half spectra; kpsi in/out. */
void REFP(update_eom_py)(void* h, void* kpsi, const void* knl, const void* knoise, double namp, double dt,
                         double eps, double lx, double ly, double lz) {
    RefState* s = (RefState*)h;
    const size_t b = REFP(state_bytes)(h);
    up(s, s->kpsi, kpsi, b);
    up(s, s->knl, knl, b);
    up(s, s->knoise, knoise, b);
    call_kernel_update_eom_py(*s->kpsi, *s->knl, *s->knoise, Float(namp), Float(dt), Float(eps), mk3(lx, ly, lz));
    down(s, s->kpsi, kpsi, b);
}

/* The 2D anisotropic-noise update (eom.hpp:16-58) on host half spectra; kpsi in/out. */
void REFP(update_eom_hpfcnoise)(void* h, void* kpsi, const void* knl, const void* n1, const void* n2,
                                const void* n3, double namp, double dt, double eps, double lx, double ly, double lz) {
    RefState* s = (RefState*)h;
    const size_t b = REFP(state_bytes)(h);
    up(s, s->kpsi, kpsi, b);
    up(s, s->knl, knl, b);
    up(s, s->knoise, n1, b);
    up(s, s->ktmp, n2, b);
    up(s, s->lpsi, n3, b);
    call_kernel_update_eom_hpfcnoise(*s->kpsi, *s->knl, *s->knoise, *s->ktmp, *s->lpsi, Float(namp), Float(dt),
                                     Float(eps), mk3(lx, ly, lz));
    down(s, s->kpsi, kpsi, b);
}

}  // extern "C"
