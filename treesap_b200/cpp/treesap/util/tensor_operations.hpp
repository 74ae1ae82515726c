// treesap-b200: compile-time unrolled tensor sums and index permutations.
// Public API of the reference util/tensor_operations.hpp:23-217. The summation order is the
// reference's (a value-initialised accumulator, then += term by term with the first index
// outermost), so FP64 results round identically.
#pragma once

#include <AMReX.H>

#include <utility>

namespace treesap {
namespace tensor {

/// Declared only for return-type deduction of f.template operator()<Is...>(); never defined.
template <typename F, int... Is>
AMREX_GPU_HOST_DEVICE constexpr auto contract_return_type(F&& f, std::integer_sequence<int, Is...>)
    -> decltype(f.template operator()<Is...>());

namespace detail {
template <int rank, int dim, typename R, typename F, int... Prefix> struct Contraction {
    template <int... Is>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE static constexpr void add(R& acc, F& f, std::integer_sequence<int, Is...>) {
        if constexpr (rank == 1) {
            ((acc += f.template operator()<Prefix..., Is>()), ...);
        } else {
            ((acc += sum<Is>(f)), ...);
        }
    }
    template <int I> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE static constexpr R sum(F& f) {
        R inner{};
        Contraction<rank - 1, dim, R, F, Prefix..., I>::add(inner, f, std::make_integer_sequence<int, dim>{});
        return inner;
    }
};
} // namespace detail

/// sum over all index tuples (a_1..a_rank) in [0, dim)^rank of f.template operator()<a_1, .., a_rank>().
template <int rank, int dim, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto contract(F&& f) {
    static_assert(rank >= 1, "contract needs at least one index");
    using R = decltype(contract_return_type(f, std::make_integer_sequence<int, rank>{}));
    R acc{};
    detail::Contraction<rank, dim, R, std::remove_reference_t<F>>::add(acc, f, std::make_integer_sequence<int, dim>{});
    return acc;
}

/// contract<rank, 3>.
template <int rank, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto contract(F&& f) {
    return contract<rank, 3>(std::forward<F>(f));
}

/// contract<1, 3>.
template <typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto contract(F&& f) {
    return contract<1, 3>(std::forward<F>(f));
}

/// (f<a,b> + f<b,a>) / 2
template <int a, int b, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto symmetrise(F&& f) {
    return 0.5 * (f.template operator()<a, b>() + f.template operator()<b, a>());
}

/// (f<a,b> - f<b,a>) / 2, and 0 without any evaluation when a == b.
template <int a, int b, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto antisymmetrise(F&& f) {
    if constexpr (a == b) {
        return 0.0;
    } else {
        return 0.5 * (f.template operator()<a, b>() - f.template operator()<b, a>());
    }
}

/// mean over the six permutations of (a, b, c).
template <int a, int b, int c, typename F> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto symmetrise(F&& f) {
    return (1.0 / 6.0) *
           (f.template operator()<a, b, c>() + f.template operator()<b, c, a>() + f.template operator()<c, a, b>() +
            f.template operator()<a, c, b>() + f.template operator()<b, a, c>() + f.template operator()<c, b, a>());
}

/// signed mean over the six permutations of (a, b, c); 0 without evaluation when two indices coincide.
template <int a, int b, int c, typename F>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto antisymmetrise(F&& f) {
    if constexpr (a == b || b == c || a == c) {
        return 0.0;
    } else {
        return (1.0 / 6.0) * (f.template operator()<a, b, c>() + f.template operator()<b, c, a>() +
                              f.template operator()<c, a, b>() - f.template operator()<a, c, b>() -
                              f.template operator()<b, a, c>() - f.template operator()<c, b, a>());
    }
}

/// mean over the three cyclic permutations of (a, b, c).
template <int a, int b, int c, typename F>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr auto cyclic_permutation_sum(F&& f) {
    return (1.0 / 3.0) *
           (f.template operator()<a, b, c>() + f.template operator()<b, c, a>() + f.template operator()<c, a, b>());
}

} // namespace tensor
} // namespace treesap
