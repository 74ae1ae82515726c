// treesap-b200: compile-time unrolled loops over an integer template parameter.
// Public API of the reference util/static_for.hpp:38-68: static_for<Start, End>(f) and
// static_for<End>(f) call f.template operator()<i>() for i = Start .. End-1 in order.
#pragma once

#include <AMReX.H>

#include <utility>

namespace treesap {

namespace detail {
template <int Start, typename F, int... Is>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr void static_for_expand(F& f, std::integer_sequence<int, Is...>) {
    (f.template operator()<Start + Is>(), ...);
}
} // namespace detail

template <int Start, int End, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr void static_for(F&& f) {
    static_assert(Start <= End, "static_for: Start must not exceed End");
    detail::static_for_expand<Start>(f, std::make_integer_sequence<int, End - Start>{});
}

template <int End, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr void static_for(F&& f) {
    static_for<0, End>(f);
}

} // namespace treesap
