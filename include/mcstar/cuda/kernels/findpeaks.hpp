// call_kernel_findpeaks of mcstar-libs cuda/kernels/findpeaks.hpp:31-63: the strict
// 26-neighbour periodic local maxima >= ths of a cubic 3D field, written as lines
// "%f %f %f %f" (x, y, z in length units, field) to peaks_outfn, then the bond-order
// table of those maxima to oorder_outfn.  Peak finding (pfc_findpeaks) and bond order
// (pfc_bond_order) both run on the GPU; the maxima are listed in increasing linear
// index (the reference's order is that of racing atomics).  Uses the caller's Float,
// Float3 and GPUArray typedefs.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "../../bond-order-analysis/bond-order.hpp"
#include "../../common/maximum_struct.hpp"
#include "../../pfc_shim.hpp"

namespace pfc_shim {

// Strict maxima: at most one per 2x2(x2) block of cells, a bound on the record count.
template <typename F>
inline Maximum<F>* find_maxima_dev(GPUArray& input, double ths, int* n) {
    const int3 e = input.real_vext();
    pfc_ctx* c = context<F>(e);
    const long long cap = (long long)((e.x + 1) / 2) * ((e.y + 1) / 2) * (e.z > 1 ? (e.z + 1) / 2 : 1) + 1;
    Maximum<F>* dev = nullptr;
    if (cudaMalloc((void**)&dev, (size_t)cap * sizeof(Maximum<F>)) != cudaSuccess) {
        fprintf(stderr, "PFCERR: cannot allocate %lld peak records\n", cap);
        exit(EXIT_FAILURE);
    }
    PFC_SHIM_CHECK(pfc_findpeaks(c, input.ptr_void(), ths, dev, (int)cap, n), c);
    return dev;
}

template <typename F>
inline void write_peaks(const std::string& fn, const Maximum<F>* dev, int n, Float3 hh) {
    std::vector<Maximum<F>> host((size_t)n);
    if (n > 0 && cudaMemcpy(host.data(), dev, (size_t)n * sizeof(Maximum<F>), cudaMemcpyDeviceToHost) != cudaSuccess) {
        fprintf(stderr, "PFCERR: peak records copy failed\n");
        exit(EXIT_FAILURE);
    }
    FILE* f = fopen(fn.c_str(), "w");
    if (!f) {
        std::cout << "output file <" << fn << "> cannot be opened for writing" << std::endl;
        return;
    }
    for (const Maximum<F>& m : host) {
        const float x0 = m.i0 * hh.x, x1 = m.i1 * hh.y, x2 = m.i2 * hh.z;
        fprintf(f, "%f %f %f %f\n", x0, x1, x2, m.field);
    }
    fclose(f);
}

}  // namespace pfc_shim

inline void call_kernel_findpeaks(GPUArray& input, std::string peaks_outfn, std::string oorder_outfn, Float3 hh,
                                  Float3 len, Float ths, Float rlim) {
    if (len.x != len.y || len.x != len.z) {
        std::cerr << "orientational mapping needs a cube" << std::endl;
        return;
    }
    int n = 0;
    Maximum<Float>* dev = pfc_shim::find_maxima_dev<Float>(input, (double)ths, &n);
    std::cerr << "found " << n << " maxima" << std::endl;
    pfc_shim::write_peaks<Float>(peaks_outfn, dev, n, hh);
    FILE* f = fopen(oorder_outfn.c_str(), "w");
    if (f) {
        int n_rows = 0;
        const std::vector<double> rows = pfc_shim::bond_rows<Float>(dev, n, (double)hh.x, (double)hh.y, (double)hh.z,
                                                                    (double)ths, (double)len.x, (double)rlim, &n_rows);
        pfc_shim::write_bond_table(f, rows, n_rows);
        fclose(f);
    } else {
        std::cout << "output file <" << oorder_outfn << "> cannot be opened for writing" << std::endl;
    }
    cudaFree(dev);
    PFC_SHIM_SYNC();
}
