// init_pot_line of mcstar-libs cuda/potentials.hpp:1-20 (host code): a 2D external
// potential, amp * s(2 pi x / sigma, 2 pi y / sigma)^power with the smooth square
// lattice s(a, b) = (cos a + cos b + 2) / 4, confined to a band |y| < sigma / 2 by two
// tanh edges; coordinates centred on the box.  Like the reference this header uses the
// caller's typedefs CPUArray and Float3, so include it after them.
#pragma once
#include <cassert>
#include <cmath>
#include <iostream>

inline double sm_square(double x, double y) { return (std::cos(x) + std::cos(y) + 2.0) / 4.0; }

inline void init_pot_line(CPUArray& arr, const Float3 l, const Float3 h, const int power, const double sigma,
                          const double amp) {
    const int3 shape = arr.real_vext();
    assert(shape.z == 1 && shape.y > 1 && shape.x > 1 && "array is not 2d");
    auto* p = arr.ptr_real();
    const double f = 2.0 * M_PI / sigma;
    for (int i1 = 0; i1 < shape.y; ++i1) {
        const double y = i1 * h.y - l.y / 2.0;
        const double band = 0.5 * (std::tanh(y + sigma / 2) + 1.0) * 0.5 * (std::tanh(-y + sigma / 2) + 1.0);
        for (int i0 = 0; i0 < shape.x; ++i0) {
            const double x = i0 * h.x - l.x / 2.0;
            p[i1 * shape.x + i0] = amp * std::pow(sm_square(f * x, f * y), power) * band;
        }
    }
    std::cout << "\"init_pot_line\" potential initialized" << std::endl;
}
