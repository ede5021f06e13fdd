// bond_order_analysis<T> with the signature of mcstar-libs
// bond-order-analysis/bond-order.hpp:4, computed on the GPU by pfc_bond_order and
// written in the reference's text table (bond-order.cpp:333-338): a header line, then
// one tab-separated row per atom above `ths` that has neighbours within `rlim`
// (minimum image in a cubic box of side `boxsize`), columns
// x y z #nb xi q4 q6 q8 w4 q4b q6b q8b w4b.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <iostream>
#include <vector>

#include "../common/maximum_struct.hpp"
#include "../pfc_shim.hpp"

namespace pfc_shim {

// bond order of n device records; rows (PFC_BOND_NCOL doubles each) returned on the host
template <typename T>
inline std::vector<double> bond_rows(const Maximum<T>* dev, int n, double h0, double h1, double h2, double ths,
                                     double boxsize, double rlim, int* n_rows) {
    pfc_ctx* c = context<T>(int3{2, 2, 2});  // bond order does not depend on the grid
    std::vector<double> rows;
    *n_rows = 0;
    if (n <= 0) return rows;
    double* drows = nullptr;
    if (cudaMalloc((void**)&drows, (size_t)n * PFC_BOND_NCOL * sizeof(double)) != cudaSuccess) {
        fprintf(stderr, "PFCERR: cannot allocate %d bond-order rows\n", n);
        exit(EXIT_FAILURE);
    }
    PFC_SHIM_CHECK(pfc_bond_order(c, dev, n, h0, h1, h2, ths, boxsize, rlim, drows, n, n_rows), c);
    rows.resize((size_t)*n_rows * PFC_BOND_NCOL);
    if (*n_rows > 0 &&
        cudaMemcpy(rows.data(), drows, rows.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        fprintf(stderr, "PFCERR: bond-order rows copy failed\n");
        exit(EXIT_FAILURE);
    }
    cudaFree(drows);
    return rows;
}

inline void write_bond_table(FILE* fp, const std::vector<double>& rows, int n_rows) {
    fprintf(fp, "# x y z #nb xi q4 q6 q8 w4 q4b q6b q8b w4b\n");
    for (int i = 0; i < n_rows; ++i) {
        const double* r = &rows[(size_t)i * PFC_BOND_NCOL];
        fprintf(fp, "%.6f\t%.6f\t%.6f\t%d\t%d\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\t%.6f\n", r[0], r[1], r[2],
                (int)r[3], (int)r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11], r[12]);
    }
    fflush(fp);
}

}  // namespace pfc_shim

// input: host records (as the reference's findpeaks produces them)
template <typename T>
inline void bond_order_analysis(Maximum<T>* input, int input_len, double h0, double h1, double h2, double _ths,
                                double _boxsize, double _rlim, FILE* fp) {
    Maximum<T>* dev = nullptr;
    if (input_len > 0) {
        if (cudaMalloc((void**)&dev, (size_t)input_len * sizeof(Maximum<T>)) != cudaSuccess ||
            cudaMemcpy(dev, input, (size_t)input_len * sizeof(Maximum<T>), cudaMemcpyHostToDevice) != cudaSuccess) {
            fprintf(stderr, "PFCERR: cannot stage %d maxima on the device\n", input_len);
            exit(EXIT_FAILURE);
        }
    }
    int n_rows = 0;
    const std::vector<double> rows = pfc_shim::bond_rows<T>(dev, input_len, h0, h1, h2, _ths, _boxsize, _rlim, &n_rows);
    if (dev) cudaFree(dev);
    pfc_shim::write_bond_table(fp, rows, n_rows);
}
