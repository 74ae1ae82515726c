// treesap-b200: centred finite-difference stencils of half-width ngrow.
//
// Weights (the formulas of the reference util/stencil_impl.hpp:56-140, n = ngrow, p = offset):
//   first : 0 at p = 0, else  sign(p) (-1)^{|p|+1} (n!)^2 / (|p| (n-|p|)! (n+|p|)!)
//   second: -2 H_{n,2} at p = 0, else  2 (-1)^{|p|+1} (n!)^2 / (p^2 (n-|p|)! (n+|p|)!)
//   third : 0 at p = 0, else  sign(p) 6 (-1)^{|p|+1} (n!)^2 (1 - p^2 H_{n,2}) / (|p|^3 (n-|p|)! (n+|p|)!)
// Each weight is the exactly representable numerator divided by the exactly representable
// denominator in double, i.e. the correctly rounded rational, as in the reference.
//
// Evaluation (reference stencil_impl.hpp:192-378): unmixed derivatives sum weighted
// differences/sums of the 2 ngrow neighbours in increasing offset order and scale by
// 1/dx^order at the end; mixed derivatives nest one-dimensional stencils. The arithmetic
// runs in the array's value type V (double for the reference's Array4<const Real>; float for
// the FP32 stage form), with the weights rounded once to V.
#pragma once

#include <AMReX.H>

#include <type_traits>

#include "cexprmath.hpp"
#include "static_for.hpp"

namespace treesap {

namespace stencil {
/// Direction shorthands: x = 0, y = 1, z = 2.
enum dir : int { x = 0, y = 1, z = 2 };
} // namespace stencil

namespace stencil_impl {
namespace weights {

template <int ngrow> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr amrex::Real first(int offset) {
    static_assert(ngrow > 0, "first derivatives need ngrow >= 1");
    using namespace cexprmath;
    const int p = offset < 0 ? -offset : offset;
    if (p == 0) return 0.0;
    const std::int64_t num = alternating_sign(p + 1) * power(factorial(ngrow), 2);
    const std::int64_t den = p * factorial(ngrow - p) * factorial(ngrow + p);
    const double w = static_cast<double>(num) / static_cast<double>(den);
    return offset > 0 ? w : -w;
}

template <int ngrow> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr amrex::Real second(int offset) {
    static_assert(ngrow > 0, "second derivatives need ngrow >= 1");
    using namespace cexprmath;
    const int p = offset < 0 ? -offset : offset;
    if (p == 0) return -2.0 * generalised_harmonic_number(ngrow, 2);
    const std::int64_t num = 2 * alternating_sign(p + 1) * power(factorial(ngrow), 2);
    const std::int64_t den = std::int64_t(p) * p * factorial(ngrow - p) * factorial(ngrow + p);
    return static_cast<double>(num) / static_cast<double>(den);
}

template <int ngrow> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr amrex::Real third(int offset) {
    static_assert(ngrow > 1, "third derivatives need ngrow >= 2");
    using namespace cexprmath;
    const int p = offset < 0 ? -offset : offset;
    if (p == 0) return 0.0;
    const std::int64_t num = 6 * alternating_sign(p + 1) * power(factorial(ngrow), 2);
    const std::int64_t den = power(p, 3) * factorial(ngrow - p) * factorial(ngrow + p);
    const double w = (1.0 - static_cast<double>(p * p) * generalised_harmonic_number(ngrow, 2)) *
                     static_cast<double>(num) / static_cast<double>(den);
    return offset > 0 ? w : -w;
}

} // namespace weights

namespace detail {

template <int d> struct Unit {
    static constexpr int x = (d == 0), y = (d == 1), z = (d == 2);
};

template <typename ArrayType> using value_t = std::remove_cv_t<ArrayType>;

// d/dx_d
template <int ngrow, int d, typename ArrayType>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE value_t<ArrayType> d1(int i, int j, int k, int comp,
                                                               const amrex::Array4<ArrayType>& arr,
                                                               const amrex::GeometryData& geom) {
    using V = value_t<ArrayType>;
    using U = Unit<d>;
    const amrex::Real gf = 1.0 / geom.CellSize(d);
    V acc = V(0);
    static_for<1, ngrow + 1>([&]<int s>() {
        constexpr V w = V(weights::first<ngrow>(s));
        acc += w * (arr(i + s * U::x, j + s * U::y, k + s * U::z, comp) -
                    arr(i - s * U::x, j - s * U::y, k - s * U::z, comp));
    });
    return V(gf) * acc;
}

// d^2/dx_d^2
template <int ngrow, int d, typename ArrayType>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE value_t<ArrayType> d2(int i, int j, int k, int comp,
                                                               const amrex::Array4<ArrayType>& arr,
                                                               const amrex::GeometryData& geom) {
    using V = value_t<ArrayType>;
    using U = Unit<d>;
    const amrex::Real gf = 1.0 / (geom.CellSize(d) * geom.CellSize(d));
    constexpr V w0 = V(weights::second<ngrow>(0));
    V acc = w0 * arr(i, j, k, comp);
    static_for<1, ngrow + 1>([&]<int s>() {
        constexpr V w = V(weights::second<ngrow>(s));
        acc += w * (arr(i + s * U::x, j + s * U::y, k + s * U::z, comp) +
                    arr(i - s * U::x, j - s * U::y, k - s * U::z, comp));
    });
    return V(gf) * acc;
}

// d^3/dx_d^3
template <int ngrow, int d, typename ArrayType>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE value_t<ArrayType> d3(int i, int j, int k, int comp,
                                                               const amrex::Array4<ArrayType>& arr,
                                                               const amrex::GeometryData& geom) {
    using V = value_t<ArrayType>;
    using U = Unit<d>;
    const amrex::Real gf = 1.0 / (geom.CellSize(d) * geom.CellSize(d) * geom.CellSize(d));
    V acc = V(0);
    static_for<1, ngrow + 1>([&]<int s>() {
        constexpr V w = V(weights::third<ngrow>(s));
        acc += w * (arr(i + s * U::x, j + s * U::y, k + s * U::z, comp) -
                    arr(i - s * U::x, j - s * U::y, k - s * U::z, comp));
    });
    return V(gf) * acc;
}

// d/dx_outer applied to an inner derivative functor g(i, j, k): first-derivative weights on
// g evaluated at the 2 ngrow neighbours along `outer`, scaled by 1/dx_outer.
template <int ngrow, int outer, typename V, typename G>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE V nest_d1(int i, int j, int k, const amrex::GeometryData& geom, G&& g) {
    using U = Unit<outer>;
    const amrex::Real gf = 1.0 / geom.CellSize(outer);
    V acc = V(0);
    static_for<1, ngrow + 1>([&]<int s>() {
        constexpr V w = V(weights::first<ngrow>(s));
        acc += w * (g(i + s * U::x, j + s * U::y, k + s * U::z) - g(i - s * U::x, j - s * U::y, k - s * U::z));
    });
    return V(gf) * acc;
}

} // namespace detail

/// Dispatch of stencil::derivative<ngrow, ArrayType, Dirs...> (one to three directions).
template <int ngrow, typename ArrayType, int... Dirs> struct derivative_impl;

template <int ngrow, typename ArrayType, int d0> struct derivative_impl<ngrow, ArrayType, d0> {
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE detail::value_t<ArrayType>
    eval(int i, int j, int k, int comp, const amrex::Array4<ArrayType>& arr, const amrex::GeometryData& geom) {
        return detail::d1<ngrow, d0>(i, j, k, comp, arr, geom);
    }
};

template <int ngrow, typename ArrayType, int d0, int d1_> struct derivative_impl<ngrow, ArrayType, d0, d1_> {
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE detail::value_t<ArrayType>
    eval(int i, int j, int k, int comp, const amrex::Array4<ArrayType>& arr, const amrex::GeometryData& geom) {
        using V = detail::value_t<ArrayType>;
        if constexpr (d0 == d1_) {
            return detail::d2<ngrow, d0>(i, j, k, comp, arr, geom);
        } else {
            return detail::nest_d1<ngrow, d0, V>(i, j, k, geom, [&](int a, int b, int c) {
                return detail::d1<ngrow, d1_>(a, b, c, comp, arr, geom);
            });
        }
    }
};

template <int ngrow, typename ArrayType, int d0, int d1_, int d2_>
struct derivative_impl<ngrow, ArrayType, d0, d1_, d2_> {
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE detail::value_t<ArrayType>
    eval(int i, int j, int k, int comp, const amrex::Array4<ArrayType>& arr, const amrex::GeometryData& geom) {
        using V = detail::value_t<ArrayType>;
        if constexpr (d0 == d1_ && d1_ == d2_) {
            return detail::d3<ngrow, d0>(i, j, k, comp, arr, geom);
        } else if constexpr (d0 == d1_ || d0 == d2_ || d1_ == d2_) {
            // one direction appears twice: d/dx_single of the unmixed second derivative along the repeated one
            constexpr int single = (d0 == d1_) ? d2_ : (d0 == d2_) ? d1_ : d0;
            constexpr int twice = (d0 == d1_) ? d0 : (d0 == d2_) ? d0 : d1_;
            return detail::nest_d1<ngrow, single, V>(i, j, k, geom, [&](int a, int b, int c) {
                return detail::d2<ngrow, twice>(a, b, c, comp, arr, geom);
            });
        } else {
            return detail::nest_d1<ngrow, d0, V>(i, j, k, geom, [&](int a, int b, int c) {
                return derivative_impl<ngrow, ArrayType, d1_, d2_>::eval(a, b, c, comp, arr, geom);
            });
        }
    }
};

} // namespace stencil_impl
} // namespace treesap
