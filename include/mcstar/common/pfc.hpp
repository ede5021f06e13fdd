// Liquid-state thermodynamics of the PFC model, as mcstar-libs common/pfc.hpp:2-7:
// chemical potential mu = dF/dpsi0 and grand potential density omega = f - mu psi0 of
// the uniform liquid, f = (1 - eps) psi0^2 / 2 + psi0^4 / 4.
#pragma once
#include <cmath>

inline double mu(double eps, double psi0) { return (1.0 - eps) * psi0 + std::pow(psi0, 3); }
inline double omega(double eps, double psi0) {
    return 0.5 * (1.0 - eps) * std::pow(psi0, 2) + 0.25 * std::pow(psi0, 4) - mu(eps, psi0) * psi0;
}
inline double omega(double eps, double psi0, double fen) { return fen - mu(eps, psi0) * psi0; }
