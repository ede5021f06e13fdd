// A host program written against the mcstar-libs source API for the other
// propagators (compiled with -I include/mcstar, linked with libpfc_b200): exponential
// conserved steps (cuda/kernels/eom-exp.hpp), then non-conserved relaxation
// (cuda/kernels/el.hpp) until the largest mode change falls below a tolerance.
//
//   driver_relax <nx> <ny> <nz> <dx> <steps> <dt> <eps> <in.npy> <outdir>
//
// Writes <outdir>/kpsi_exp.npy after the exponential steps and <outdir>/kpsi_el.npy
// after the relaxation; prints "iters <n> change <last max change>".
#include <cuda/array_abstraction.hpp>
#include <cuda/cufft_wrapper.hpp>
#include <common/cu_error.hpp>

#include <cstdlib>
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
#include <cuda/kernels/eom-exp.hpp>
#include <cuda/kernels/el.hpp>
#include <cuda/kernels/el-exp.hpp>
#include <cuda/kernels/psi3_split.hpp>

int main(int argc, char* argv[]) {
    if (argc != 10) {
        std::cerr << "usage: " << argv[0] << " nx ny nz dx steps dt eps in.npy outdir" << std::endl;
        return EXIT_FAILURE;
    }
    CUERR(cudaSetDevice(0));
    const int3 shape{atoi(argv[1]), atoi(argv[2]), atoi(argv[3])};
    const Float dx = (Float)atof(argv[4]);
    const int steps = atoi(argv[5]);
    const Float dt = (Float)atof(argv[6]), eps = (Float)atof(argv[7]);
    const std::string in(argv[8]), outdir(argv[9]);
    const Float3 lens{shape.x * dx, shape.y * dx, shape.z == 1 ? (Float)1 : shape.z * dx};

    CPUArray host(shape);
    host.load(in);
    GPUArray psi(host), kpsi(shape), tmp(shape), knl(shape), kop(shape);
    PlanR2C r2c(shape);
    PlanC2R c2r(shape);
    r2c.execute(psi, kpsi);

    call_kernel_init_eom_op(kop, dt, eps, lens);
    for (int s = 0; s < steps; ++s) {
        kpsi >> tmp;
        c2r.execute(tmp, psi);
        call_kernel_psi3_split(psi, nullptr, (Float)0, true);
        r2c.execute(psi, knl);
        call_kernel_update_eom(kop, kpsi, knl, (Float)0, dt, eps, lens);
    }
    CPUArray out(shape);
    kpsi >> out;
    out.save<Array::AsCmpl>(outdir + "/kpsi_exp.npy");

    Float change = 0;
    int it = 0;
    for (; it < 200; ++it) {
        kpsi >> tmp;
        c2r.execute(tmp, psi);
        call_kernel_psi3_split(psi, nullptr, (Float)0, true);
        r2c.execute(psi, knl);
        change = call_kernel_update_el(kpsi, knl, dt, eps, lens);
        if (change < (Float)1e-3) break;
    }
    kpsi >> out;
    out.save<Array::AsCmpl>(outdir + "/kpsi_el.npy");
    std::cout << "iters " << it << " change " << change << std::endl;
    return EXIT_SUCCESS;
}
