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

#include "stencil_impl.hpp"

namespace treesap {
namespace stencil {

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

} // namespace stencil
} // namespace treesap
