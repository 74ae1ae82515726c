// treesap-b200: public stencil operators (reference util/stencil.hpp:42-104).
//
//   stencil::derivative<ngrow, ArrayType, Dirs...>(arr, comp, idx, geom)
//       centred first/second/third derivative of arr(., comp) at idx (1 to 3 directions).
//   stencil::kreiss_oliger<order, dir>(arr, comp, idx, geom)
//       D_KO = (-1)^{r+1} dx^{2r-1} 2^{-2r} (D+ D-)^r f
//            = -(1/dx) 2^{-2r} sum_{m=-r..r} (-1)^m C(2r, r+m) f_m,
//       accumulated as -C(2r,r) f_0 + sum_{s=1..r} -(-1)^s C(2r, r+s) (f_s + f_-s),
//       then scaled by 2^{-2r} and by 1/dx (reference order).
// kreiss_oliger also accepts (idx, comp, arr, geom), the argument order used by the
// reference's KODecorator (pde-model/rhs-decorators/KODecorator.hpp:64-66).
#pragma once

#include <AMReX.H>

#include <cmath>
#include <type_traits>

#include "stencil_impl.hpp"

namespace treesap {
namespace stencil {

namespace detail {
/// a * b + c rounded once, in the value type (double or float), on host and device.
template <typename V> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE V fma_rn(V a, V b, V c) {
#if defined(__CUDA_ARCH__)
    if constexpr (std::is_same_v<V, float>)
        return __fmaf_rn(a, b, c);
    else
        return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
} // namespace detail

template <int ngrow, typename ArrayType, int... Dirs>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE std::remove_cv_t<ArrayType>
derivative(const amrex::Array4<ArrayType>& arr, int comp, const amrex::IntVect& idx, const amrex::GeometryData& geom) {
    static_assert(((Dirs >= 0 && Dirs <= 2) && ...), "derivative directions must be 0, 1 or 2");
    static_assert(sizeof...(Dirs) >= 1 && sizeof...(Dirs) <= 3, "first to third derivatives only");
    return stencil_impl::derivative_impl<ngrow, ArrayType, Dirs...>::eval(idx[0], idx[1], idx[2], comp, arr, geom);
}

template <int order, int d, typename ArrayType>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE std::remove_cv_t<ArrayType>
kreiss_oliger(const amrex::Array4<ArrayType>& arr, int comp, const amrex::IntVect& idx,
              const amrex::GeometryData& geom) {
    static_assert(order > 0, "Kreiss-Oliger order must be positive");
    using V = std::remove_cv_t<ArrayType>;
    using U = stencil_impl::detail::Unit<d>;
    using namespace cexprmath;
    const int i = idx[0], j = idx[1], k = idx[2];
    constexpr V c0 = V(-binom(2 * order, order));
    constexpr double norm = 1.0 / static_cast<double>(power(2, 2 * order));
    const amrex::Real gf = 1.0 / geom.CellSize(d);
    V acc = c0 * arr(i, j, k, comp);
    static_for<1, order + 1>([&]<int s>() {
        constexpr V c = V(-alternating_sign(s) * binom(2 * order, order + s));
        acc += c * (arr(i + s * U::x, j + s * U::y, k + s * U::z, comp) +
                    arr(i - s * U::x, j - s * U::y, k - s * U::z, comp));
    });
    // one multiply by norm * gf: norm is a power of two, so this rounds exactly like
    // (acc * norm) * gf
    return acc * V(norm * gf);
}

template <int order, int d, typename ArrayType>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE std::remove_cv_t<ArrayType>
kreiss_oliger(const amrex::IntVect& idx, int comp, const amrex::Array4<ArrayType>& arr,
              const amrex::GeometryData& geom) {
    return kreiss_oliger<order, d, ArrayType>(arr, comp, idx, geom);
}

/// base + strength * (D_KO^x + D_KO^y + D_KO^z) arr(., comp): the three directions of
/// kreiss_oliger in one pass (treesap-b200 extension, used by KODecorator). Mathematically the
/// same sum, reassociated for fewer operations: per direction the off-centre binomial terms
/// acc_d = sum_s c_s (f_s + f_-s); then
///   base + s0 f_0 + s_x acc_x + s_y acc_y + s_z acc_z,
/// with s_d = strength 2^{-2r} / dx_d and s0 = c_0 (s_x + s_y + s_z) (loop-invariant factors).
/// It differs from the direction-by-direction sum only by rounding (a few ulp). Every
/// accumulation is an explicit fused multiply-add, so the rounding does not depend on how the
/// compiler contracts the surrounding code (models that add the same terms in the same order
/// agree bitwise).
template <int order, typename ArrayType, typename V = std::remove_cv_t<ArrayType>>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE V kreiss_oliger_added(V base, const amrex::Array4<ArrayType>& arr, int comp,
                                                               const amrex::IntVect& idx,
                                                               const amrex::GeometryData& geom, amrex::Real strength) {
    static_assert(order > 0, "Kreiss-Oliger order must be positive");
    using namespace cexprmath;
    const int i = idx[0], j = idx[1], k = idx[2];
    constexpr double c0 = -double(binom(2 * order, order));
    constexpr double norm = 1.0 / static_cast<double>(power(2, 2 * order));
    const amrex::Real sx = strength * norm / geom.CellSize(0), sy = strength * norm / geom.CellSize(1),
                      sz = strength * norm / geom.CellSize(2);
    const V s0 = V(c0 * (sx + sy + sz));
    V acc[3];
    static_for<0, 3>([&]<int d>() {
        using U = stencil_impl::detail::Unit<d>;
        static_for<1, order + 1>([&]<int s>() {
            constexpr V c = V(-alternating_sign(s) * binom(2 * order, order + s));
            const V p = arr(i + s * U::x, j + s * U::y, k + s * U::z, comp) +
                        arr(i - s * U::x, j - s * U::y, k - s * U::z, comp);
            if constexpr (s == 1)
                acc[d] = c * p;
            else
                acc[d] = detail::fma_rn(c, p, acc[d]);
        });
    });
    V r = detail::fma_rn(s0, V(arr(i, j, k, comp)), base);
    r = detail::fma_rn(V(sx), acc[0], r);
    r = detail::fma_rn(V(sy), acc[1], r);
    r = detail::fma_rn(V(sz), acc[2], r);
    return r;
}

} // namespace stencil
} // namespace treesap
