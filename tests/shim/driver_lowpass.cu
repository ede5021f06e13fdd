// A host program written against the mcstar-libs source API for the 2D spectral low-pass
// (compiled with -I include/mcstar, linked with libpfc_b200): the R2C of a field, the
// Gaussian filter (cuda/kernels/gaussian.hpp) and calc_amplitude_lowpass
// (cuda/kernels/lowpass.hpp), which writes the LOWPASS dump and leaves the amplitude in
// the host array.
//
//   driver_lowpass <nx> <ny> <dx> <divs_per_sigma> <in.npy> <outdir>
//
// Writes <outdir>/lowpass.gz and <outdir>/amplitude.npy.
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
#include <cuda/kernels/gaussian.hpp>
#include <cuda/kernels/lowpass.hpp>

int main(int argc, char* argv[]) {
    if (argc != 7) {
        std::cerr << "usage: " << argv[0] << " nx ny dx divs_per_sigma in.npy outdir" << std::endl;
        return EXIT_FAILURE;
    }
    CUERR(cudaSetDevice(0));
    const int3 shape{atoi(argv[1]), atoi(argv[2]), 1};
    const Float dx = (Float)atof(argv[3]), dps = (Float)atof(argv[4]);
    const std::string in(argv[5]), outdir(argv[6]);
    const Float3 lens{shape.x * dx, shape.y * dx, (Float)1};
    const Float3 hh{dx, dx, (Float)1};

    CPUArray host(shape);
    host.load(in);
    GPUArray psi(host), spectrum(shape), aux(shape), kgauss(shape);
    PlanR2C r2c(shape);
    PlanC2R c2r(shape);
    r2c.execute(psi, spectrum);
    call_kernel_gaussian_init(kgauss, lens, hh, dps);
    calc_amplitude_lowpass(r2c, c2r, spectrum, aux, kgauss, host, lens, outdir + "/lowpass.gz");
    host.save<Array::AsReal>(outdir + "/amplitude.npy");
    return EXIT_SUCCESS;
}
