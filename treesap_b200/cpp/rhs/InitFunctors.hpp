// Built-in initial-condition functors (InitConcept, reference pde-model/PDEModelConcepts.hpp:96-108),
// evaluated by the integrator at cell centres lo + (i + 1/2) dx (reference SingleLevelIntegrator.hpp:84-87).
// Trivially copyable: parameters are held in fixed-size arrays.
#pragma once

#include "pde-model/PDEModelConcepts.hpp"

#include <cmath>

namespace tsb {

/// Sum of Gaussian pulses:  u_c(x) = sum_{p : comp_p == c} A_p exp(-|x - c_p|^2 / w_p^2).
template <int ncomp_> struct GaussianSumInit {
    static constexpr int ncomp = ncomp_;
    static constexpr int max_pulses = 16;

    int npulses = 0;
    int comp[max_pulses] = {};
    double amp[max_pulses] = {}, width[max_pulses] = {};
    double cx[max_pulses] = {}, cy[max_pulses] = {}, cz[max_pulses] = {};

    template <int c>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real operator()(amrex::Real x, amrex::Real y,
                                                                    amrex::Real z) const {
        amrex::Real v = 0.0;
        for (int p = 0; p < npulses; ++p) {
            if (comp[p] != c) continue;
            const amrex::Real dx = x - cx[p], dy = y - cy[p], dz = z - cz[p];
            v += amp[p] * std::exp(-(dx * dx + dy * dy + dz * dz) / (width[p] * width[p]));
        }
        return v;
    }
};

/// Sum of Fourier modes on the unit-period box:  u_c(x) = sum_{m : comp_m == c} A_m cos(2 pi k_m . x + theta_m).
template <int ncomp_> struct FourierSumInit {
    static constexpr int ncomp = ncomp_;
    static constexpr int max_modes = 256;

    int nmodes = 0;
    int comp[max_modes] = {};
    double amp[max_modes] = {}, phase[max_modes] = {};
    double kx[max_modes] = {}, ky[max_modes] = {}, kz[max_modes] = {};

    template <int c>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real operator()(amrex::Real x, amrex::Real y,
                                                                    amrex::Real z) const {
        constexpr amrex::Real two_pi = 6.283185307179586476925286766559;
        amrex::Real v = 0.0;
        for (int m = 0; m < nmodes; ++m) {
            if (comp[m] != c) continue;
            v += amp[m] * std::cos(two_pi * (kx[m] * x + ky[m] * y + kz[m] * z) + phase[m]);
        }
        return v;
    }
};

/// Absorbing-layer damping profiles s -> profile(s) with profile(0) = 0 and profile(1) = 1
/// (ABLProfileConcept, reference pde-model/rhs-decorators/ABLDecorator.hpp:24-29).
struct QuadraticProfile {
    constexpr amrex::Real operator()(amrex::Real s) const { return s * s; }
    /// The same profile as a function of s^2 (the B200 front end's ABLDecorator then needs no
    /// square root and no branch; the reference calls operator() only).
    constexpr amrex::Real of_square(amrex::Real s2) const { return s2; }
};
struct LinearProfile {
    constexpr amrex::Real operator()(amrex::Real s) const { return s; }
};

} // namespace tsb
