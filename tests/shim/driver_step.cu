// A host program written against the mcstar-libs source API (compiled with
// -I include/mcstar, linked with libpfc_b200): the per-step loop of the reference's
// drivers -- copy psi^, C2R, psi3_split (normalised), R2C, [fill_kspace], update_eom --
// then the free energy, the peak list and the bond-order table.
//
//   driver_step <nx> <ny> <nz> <dx> <steps> <dt> <eps> <namp> <seed> <in.npy> <outdir>
//
// Writes <outdir>/kpsi.npy (final half spectrum), <outdir>/peaks.txt,
// <outdir>/bond.txt (3D only) and prints "F <free energy>" and "ms <device time>".
#include <cuda/array_abstraction.hpp>
#include <cuda/cufft_wrapper.hpp>
#include <cuda/noise.hpp>
#include <cuda/cutiming.hpp>
#include <common/cu_error.hpp>
#include <common/pfc.hpp>

#include <cmath>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <string>

typedef FLOAT Float;
typedef Array::CPUArray<Float> CPUArray;
typedef Array::GPUArray<Float> GPUArray;
typedef FFT::CufftPlan<Float, FFT::R2C> PlanR2C;
typedef FFT::CufftPlan<Float, FFT::C2R> PlanC2R;
typedef typename std::conditional<sizeof(Float) == 4, float2, double2>::type Float2;
typedef typename std::conditional<sizeof(Float) == 4, float3, double3>::type Float3;

#include <cuda/kernels/common.hpp>
#include <cuda/kernels/eom.hpp>
#include <cuda/kernels/findpeaks.hpp>
#include <cuda/kernels/findpeaks_2d.hpp>
#include <cuda/kernels/norm.hpp>
#include <cuda/kernels/psi3_split.hpp>

int main(int argc, char* argv[]) {
    if (argc != 12) {
        std::cerr << "usage: " << argv[0] << " nx ny nz dx steps dt eps namp seed in.npy outdir" << std::endl;
        return EXIT_FAILURE;
    }
    CUERR(cudaSetDevice(0));
    const int3 shape{atoi(argv[1]), atoi(argv[2]), atoi(argv[3])};
    const Float dx = (Float)atof(argv[4]);
    const int steps = atoi(argv[5]);
    const Float dt = (Float)atof(argv[6]), eps = (Float)atof(argv[7]), namp = (Float)atof(argv[8]);
    const unsigned long long seed = strtoull(argv[9], nullptr, 10);
    const std::string in(argv[10]), outdir(argv[11]);
    const Float3 hh{dx, dx, dx};
    const Float3 lens{shape.x * dx, shape.y * dx, shape.z == 1 ? (Float)1 : shape.z * dx};

    CPUArray host(shape);
    host.load(in);
    GPUArray psi(host), kpsi(shape), tmp(shape), knl(shape), knoise(shape), lpsi(shape);
    PlanR2C r2c(shape);
    PlanC2R c2r(shape);
    NoiseHostApi<Float> noise(seed);
    const double psi0 = 0.0;
    const Float m = (Float)mu((double)eps, psi0);

    r2c.execute(psi, kpsi);
    TimeAcc t;
    t.start();
    for (int s = 0; s < steps; ++s) {
        kpsi >> tmp;
        c2r.execute(tmp, psi);
        call_kernel_psi3_split(psi, nullptr, m, true);
        r2c.execute(psi, knl);
        if (namp != 0) {
            noise.fill_kspace(knoise);
            call_kernel_update_eom(kpsi, knl, knoise, namp, dt, eps, lens);
        } else {
            call_kernel_update_eom(kpsi, knl, namp, dt, eps, lens);
        }
    }
    t.stop();

    CPUArray out(shape);
    kpsi >> out;
    out.save<Array::AsCmpl>(outdir + "/kpsi.npy");

    // free energy of the final state: L^psi^ from a zero-length update, both fields to
    // real space, normalised, then h^3 sum f
    kpsi >> tmp;
    call_kernel_update_eom_with_fen(tmp, knl, knoise, (Float)0, (Float)0, eps, lens);
    c2r.execute(knoise, lpsi);
    call_kernel_norm(lpsi);
    c2r.execute(kpsi, psi);
    call_kernel_norm(psi);
    const float F = call_kernel_calc_fen(psi, lpsi, hh);
    std::cout << std::setprecision(9) << "F " << F << std::endl;
    std::cout << "ms " << t << std::endl;

    c2r.execute(kpsi, psi);
    call_kernel_norm(psi);
    if (shape.z == 1)
        call_kernel_findpeaks_2d(psi, outdir + "/peaks.txt", hh, lens, (Float)0);
    else
        call_kernel_findpeaks(psi, outdir + "/peaks.txt", outdir + "/bond.txt", hh, lens, (Float)0, (Float)8.3);
    return EXIT_SUCCESS;
}
