// Variable-speed scalar wave system and its discrete adjoint, written as treesap user models
// (RHSConcept) so the fused stage kernels evaluate them like any other model.
//
// The speed field travels with the state as a constant component: u = {phi, pi, c2},
//   forward   L(c2):  phi_t = pi + s K phi,          pi_t = c2 D phi + s K pi,        c2_t = 0
// with D = sum_a D2_aa (centred, half-width ngrow), K = sum_a KO_a (Kreiss-Oliger of order
// ngrow) and s the dissipation strength. On a periodic grid D and K are symmetric matrices,
// so the transpose of the (phi, pi) block is
//   adjoint   L^T:    phibar_t = s K phibar + D (c2 pibar),   pibar_t = phibar + s K pibar
// and RK4 applied to L^T is the transpose of RK4 applied to L (both are the polynomial
// 1 + z + z^2/2 + z^3/6 + z^4/24 of dt L). The tangent-linear system carries the
// perturbation alongside the state, u = {phi, pi, c2, dphi, dpi, dc2}:
//   dphi_t = dpi + s K dphi,   dpi_t = c2 D dphi + dc2 D phi + s K dpi.
// The forward model performs the same operations in the same order as
// KODecorator<WaveRHS<ngrow, FieldSpeed>> (WaveRHS.hpp), so both give identical results.
#pragma once

#include "pde-model/PDEModelConcepts.hpp"
#include "util/static_for.hpp"
#include "util/stencil.hpp"

namespace tsb {

namespace detail {
/// base + s sum_a KO_a of component n in the one-pass form, which is KODecorator's
/// arithmetic for models of at most 4 components (so the 3-component forward model is bitwise
/// the 2-component library model), or base when s = 0.
template <int G, typename T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T with_ko(T base, const amrex::Array4<const T>& arr, int n,
                                                   const amrex::IntVect& idx, const amrex::GeometryData& geom,
                                                   amrex::Real s) {
    return s > 0.0 ? treesap::stencil::kreiss_oliger_added<G>(base, arr, n, idx, geom, s) : base;
}

/// sum_a D2_aa of component n (WaveRHS's contraction order).
template <int G, typename T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T lap(const amrex::Array4<const T>& arr, int n, const amrex::IntVect& idx,
                                               const amrex::GeometryData& geom) {
    using namespace treesap::stencil;
    T l = T(0);
    treesap::static_for<3>([&]<int a>() { l += derivative<G, const T, a, a>(arr, n, idx, geom); });
    return l;
}

/// sum_a D2_aa of the product of components m and n (the same weights as lap).
template <int G, typename T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T lap_of_product(const amrex::Array4<const T>& arr, int m, int n,
                                                          const amrex::IntVect& idx, const amrex::GeometryData& geom) {
    using namespace treesap::stencil_impl;
    const int i = idx[0], j = idx[1], k = idx[2];
    auto f = [&](int a, int b, int c) { return arr(a, b, c, m) * arr(a, b, c, n); };
    T l = T(0);
    treesap::static_for<3>([&]<int d>() {
        using U = treesap::stencil_impl::detail::Unit<d>;
        const amrex::Real gf = 1.0 / (geom.CellSize(d) * geom.CellSize(d));
        constexpr T w0 = T(weights::second<G>(0));
        T acc = w0 * f(i, j, k);
        treesap::static_for<1, G + 1>([&]<int s>() {
            constexpr T w = T(weights::second<G>(s));
            acc += w * (f(i + s * U::x, j + s * U::y, k + s * U::z) + f(i - s * U::x, j - s * U::y, k - s * U::z));
        });
        l += T(gf) * acc;
    });
    return l;
}
} // namespace detail

/// Forward model {phi, pi, c2}.
template <int ngrow_> struct WaveC2RHS {
    static constexpr int ncomp = 3;
    static constexpr int ngrow = ngrow_;
    static constexpr bool is_affine_autonomous = true;
    struct Workspace {};
    amrex::Real ko_strength = 0.0;

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        if constexpr (comp == 2) {
            return T(0);
        } else {
            T base;
            if constexpr (comp == 0)
                base = arr(idx, 1);
            else
                base = arr(idx, 2) * detail::lap<ngrow>(arr, 0, idx, geom);
            return detail::with_ko<ngrow>(base, arr, comp, idx, geom, ko_strength);
        }
    }
};

/// Adjoint model {phibar, pibar, c2}: the transpose of WaveC2RHS's (phi, pi) block.
template <int ngrow_> struct WaveC2AdjointRHS {
    static constexpr int ncomp = 3;
    static constexpr int ngrow = ngrow_;
    static constexpr bool is_affine_autonomous = true;
    struct Workspace {};
    amrex::Real ko_strength = 0.0;

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        if constexpr (comp == 2) {
            return T(0);
        } else {
            T base;
            if constexpr (comp == 0)
                base = detail::lap_of_product<ngrow>(arr, 2, 1, idx, geom);
            else
                base = arr(idx, 0);
            return detail::with_ko<ngrow>(base, arr, comp, idx, geom, ko_strength);
        }
    }
};

/// {D phi, 0, 0}: the Laplacian of a forward stage argument, for the speed gradient.
template <int ngrow_> struct WaveC2LaplacianRHS {
    static constexpr int ncomp = 3;
    static constexpr int ngrow = ngrow_;
    struct Workspace {};

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        if constexpr (comp == 0)
            return detail::lap<ngrow>(arr, 0, idx, geom);
        else
            return T(0);
    }
};

/// {D phi, 0} of a two-component field {phi, pi} (or of its FP32-stage registers k0, d1, d2):
/// the Laplacian behind the FP32-stage form of the speed gradient.
template <int ngrow_> struct WaveLaplacianRHS {
    static constexpr int ncomp = 2;
    static constexpr int ngrow = ngrow_;
    struct Workspace {};

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        if constexpr (comp == 0)
            return detail::lap<ngrow>(arr, 0, idx, geom);
        else
            return T(0);
    }
};

/// Adjoint model {phibar, pibar} with the speed as a coefficient field instead of a state
/// component: phibar_t = s K phibar + D (c2 pibar), pibar_t = phibar + s K pibar, c2 read from a
/// device array of the valid cells (x fastest) with periodic wrap-around at the neighbour taps.
/// Linear in the state, so it also runs in the FP32-stage RK4 form (whose stage differences
/// would lose a coefficient carried as a state component).
template <int ngrow_> struct WaveAdjointSpeedRHS {
    static constexpr int ncomp = 2;
    static constexpr int ngrow = ngrow_;
    static constexpr bool is_affine_autonomous = true;
    struct Workspace {};
    const double* c2 = nullptr;
    int n[3] = {0, 0, 0};
    amrex::Real ko_strength = 0.0;

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        T base;
        if constexpr (comp == 0) {
            using namespace treesap::stencil_impl;
            const int i = idx[0], j = idx[1], k = idx[2];
            auto wrap = [](int a, int m) { return a < 0 ? a + m : (a >= m ? a - m : a); };
            auto f = [&](int a, int b, int c) {
                const long long q = wrap(a, n[0]) + (long long)n[0] * (wrap(b, n[1]) + (long long)n[1] * wrap(c, n[2]));
                return T(c2[q]) * arr(a, b, c, 1);
            };
            base = T(0);
            treesap::static_for<3>([&]<int d>() {
                using U = treesap::stencil_impl::detail::Unit<d>;
                const amrex::Real gf = 1.0 / (geom.CellSize(d) * geom.CellSize(d));
                constexpr T w0 = T(weights::second<ngrow>(0));
                T acc = w0 * f(i, j, k);
                treesap::static_for<1, ngrow + 1>([&]<int s>() {
                    constexpr T w = T(weights::second<ngrow>(s));
                    acc += w * (f(i + s * U::x, j + s * U::y, k + s * U::z) +
                                f(i - s * U::x, j - s * U::y, k - s * U::z));
                });
                base += T(gf) * acc;
            });
        } else {
            base = arr(idx, 0);
        }
        return detail::with_ko<ngrow>(base, arr, comp, idx, geom, ko_strength);
    }
};

/// Tangent-linear model {phi, pi, c2, dphi, dpi, dc2}.
template <int ngrow_> struct WaveC2TangentRHS {
    static constexpr int ncomp = 6;
    static constexpr int ngrow = ngrow_;
    struct Workspace {};
    amrex::Real ko_strength = 0.0;

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        if constexpr (comp == 2 || comp == 5) {
            return T(0);
        } else {
            T base;
            if constexpr (comp == 0)
                base = arr(idx, 1);
            else if constexpr (comp == 1)
                base = arr(idx, 2) * detail::lap<ngrow>(arr, 0, idx, geom);
            else if constexpr (comp == 3)
                base = arr(idx, 4);
            else
                base = arr(idx, 2) * detail::lap<ngrow>(arr, 3, idx, geom) +
                       arr(idx, 5) * detail::lap<ngrow>(arr, 0, idx, geom);
            return detail::with_ko<ngrow>(base, arr, comp, idx, geom, ko_strength);
        }
    }
};

} // namespace tsb
