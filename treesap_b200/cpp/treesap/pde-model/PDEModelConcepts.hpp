// treesap-b200: the plugin interface of a PDE model (the drop-in boundary).
//
// Same concepts as the reference pde-model/PDEModelConcepts.hpp:44-139:
//   RHSConcept     trivially copyable; static ncomp > 0, ngrow >= 0; default-constructible
//                  Workspace; template<int comp> operator()(IntVect, Real time,
//                  const Array4<const Real>&, const GeometryData&, Workspace&) const -> Real
//                  for every comp in [0, ncomp).
//   BCConcept      trivially copyable; ncomp, ngrow; operator()(const IntVect&, const Array4<Real>&,
//                  int dcomp, int numcomp, const GeometryData&, Real time, const BCRec*, int bcomp,
//                  int orig_comp) const -> void.
//   InitConcept    trivially copyable; ncomp; template<int comp> operator()(Real x, Real y, Real z) const.
//   PDEModelConcept the getters get_rhs/get_init/get_bc/get_bc_recs/get_geometry/get_comp_names/dt_hint.
//
// Extension (not in the reference): AffineRHSConcept marks right-hand sides that may run in
// the FP32-stage RK4 form: F(u) = L u + f0 with L linear, f0 independent of u and time,
// evaluable on Array4<const float>, and exposing L either as `linear_part()` or (when
// f0 = 0) as the functor itself.
#pragma once

#include <AMReX.H>

#include <concepts>
#include <string>
#include <type_traits>
#include <utility>

namespace treesap {

namespace detail {
/// operator()<I> of F is callable with the RHS signature on Array4<const V> and returns something convertible to V.
template <typename F, int I, typename V>
concept RHSComponentCallable =
    requires(const F& f, const amrex::IntVect idx, amrex::Real time, const amrex::Array4<const V>& arr,
             const amrex::GeometryData& geom, typename F::Workspace& ws) {
        { f.template operator()<I>(idx, time, arr, geom, ws) } -> std::convertible_to<V>;
    };
template <typename F, typename V, typename Seq> struct AllComponentsCallable;
template <typename F, typename V, int... Is> struct AllComponentsCallable<F, V, std::integer_sequence<int, Is...>> {
    static constexpr bool value = (RHSComponentCallable<F, Is, V> && ...);
};
} // namespace detail

template <typename F>
concept RHSConcept = std::is_trivially_copyable_v<F> && requires {
    typename std::integral_constant<int, F::ncomp>;
    typename std::integral_constant<int, F::ngrow>;
    requires F::ncomp > 0;
    requires F::ngrow >= 0;
    typename F::Workspace;
} && std::is_default_constructible_v<typename F::Workspace> &&
                     detail::AllComponentsCallable<F, amrex::Real, std::make_integer_sequence<int, F::ncomp>>::value;

template <typename F>
concept BCConcept = std::is_trivially_copyable_v<F> && requires {
    typename std::integral_constant<int, F::ncomp>;
    typename std::integral_constant<int, F::ngrow>;
    requires F::ncomp > 0;
    requires F::ngrow >= 0;
} && requires(const F& t, const amrex::IntVect& iv, const amrex::Array4<amrex::Real>& dest, int dcomp, int numcomp,
              const amrex::GeometryData& geom, amrex::Real time, const amrex::BCRec* bcr, int bcomp, int orig_comp) {
    { t(iv, dest, dcomp, numcomp, geom, time, bcr, bcomp, orig_comp) } -> std::same_as<void>;
};

template <typename F>
concept InitConcept = std::is_trivially_copyable_v<F> && requires {
    typename std::integral_constant<int, F::ncomp>;
    requires F::ncomp > 0;
} && requires(const F& f, amrex::Real x, amrex::Real y, amrex::Real z) {
    { f.template operator()<0>(x, y, z) } -> std::convertible_to<amrex::Real>;
};

template <typename M>
concept PDEModelConcept = requires {
    typename std::integral_constant<int, M::ncomp>;
    typename std::integral_constant<int, M::ngrow>;
    requires M::ncomp > 0;
    requires M::ngrow >= 0;
    typename M::rhs_t;
    typename M::init_t;
    typename M::bc_t;
} && requires(M m) {
    requires RHSConcept<typename M::rhs_t>;
    { m.get_rhs() } -> std::same_as<const typename M::rhs_t&>;
    requires InitConcept<typename M::init_t>;
    { m.get_init() } -> std::same_as<const typename M::init_t&>;
    requires BCConcept<typename M::bc_t>;
    { m.get_bc() } -> std::same_as<const typename M::bc_t&>;
    { m.get_bc_recs() } -> std::convertible_to<const amrex::Vector<amrex::BCRec>&>;
    { m.get_geometry() } -> std::same_as<const amrex::Geometry&>;
    { m.get_comp_names() } -> std::convertible_to<amrex::Vector<std::string>>;
    { m.dt_hint() } -> std::convertible_to<amrex::Real>;
};

// ------------------------------------------------------------------ FP32-stage extension

/// True when F declares `static constexpr bool is_affine_autonomous = true`.
template <typename F> constexpr bool is_affine_autonomous_v = [] {
    if constexpr (requires { F::is_affine_autonomous; }) {
        return bool(F::is_affine_autonomous);
    } else {
        return false;
    }
}();

/// The linear part L of an affine right-hand side (the functor itself when it has no offset).
template <typename F> AMREX_GPU_HOST_DEVICE constexpr auto linear_part_of(const F& f) {
    if constexpr (requires { f.linear_part(); }) {
        return f.linear_part();
    } else {
        return f;
    }
}

template <typename F>
concept AffineRHSConcept =
    RHSConcept<F> && is_affine_autonomous_v<F> &&
    detail::AllComponentsCallable<decltype(linear_part_of(std::declval<const F&>())), float,
                                  std::make_integer_sequence<int, F::ncomp>>::value;

} // namespace treesap
