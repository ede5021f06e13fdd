// call_kernel_findpeaks_2d of mcstar-libs cuda/kernels/findpeaks_2d.hpp:29-56: the
// strict 8-neighbour periodic local maxima >= ths of a 2D field, written as lines
// "%f %f %f %f" (x, y, z = 0, field).  pfc_findpeaks on the GPU; maxima in increasing
// linear index.  Uses the caller's Float, Float3 and GPUArray typedefs.
#pragma once
#include <iostream>
#include <string>

#include "findpeaks.hpp"

inline void call_kernel_findpeaks_2d(GPUArray& input, std::string peaks_outfn, Float3 hh, Float3 len, Float ths) {
    (void)len;
    const int3 shape = input.real_vext();
    if (!(shape.x > 1 && shape.y > 1 && shape.z == 1)) {
        std::cerr << "input not a 2d array" << std::endl;
        return;
    }
    int n = 0;
    Maximum<Float>* dev = pfc_shim::find_maxima_dev<Float>(input, (double)ths, &n);
    std::cerr << "found " << n << " maxima" << std::endl;
    pfc_shim::write_peaks<Float>(peaks_outfn, dev, n, hh);
    cudaFree(dev);
    PFC_SHIM_SYNC();
}
