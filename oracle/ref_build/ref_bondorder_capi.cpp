/* ORACLE / TEST INFRASTRUCTURE ONLY.
 * C entry points around the reference's own bond-order analysis
 * (bond-order-analysis/bond-order.cpp:289-349, header bond-order.hpp:4) so that
 * Python tests can call the unmodified reference through ctypes.  The reference
 * source is compiled where it lies (see oracle/Makefile); nothing is copied. */
#include <cstdio>
#include <common/maximum_struct.hpp>
#include <bond-order-analysis/bond-order.hpp>

extern "C" int ref_bond_order_f32(const void* maxima, int n, double h0, double h1, double h2,
                                  double ths, double boxsize, double rlim, const char* out_path) {
    FILE* fp = std::fopen(out_path, "w");
    if (!fp) return 1;
    bond_order_analysis<float>((Maximum<float>*)maxima, n, h0, h1, h2, ths, boxsize, rlim, fp);
    std::fclose(fp);
    return 0;
}

extern "C" int ref_bond_order_f64(const void* maxima, int n, double h0, double h1, double h2,
                                  double ths, double boxsize, double rlim, const char* out_path) {
    FILE* fp = std::fopen(out_path, "w");
    if (!fp) return 1;
    bond_order_analysis<double>((Maximum<double>*)maxima, n, h0, h1, h2, ths, boxsize, rlim, fp);
    std::fclose(fp);
    return 0;
}
