// treesap-b200: compile-time tensor views onto a range of Array4 components.
//
// Public API of the reference pde-model/tensor-alias/TensorAliasBase.hpp:44-287:
//   * CRTP base TensorAliasBase<Derived, comp_base, ncomp, rank, dim, ArrayType>, an aggregate
//     whose only data member is `const amrex::Array4<ArrayType>& arr` (so `Alias a{{arr}};` works);
//   * static constexpr comp_base, ncomp, rank, dim, next; contains(), get_absolute(),
//     restore_absolute(); element access operator()(i,j,k,indices) / (IntVect, indices);
//     load() into a register-resident Temporary;
//   * concept TensorAliasImplementation with the compile-time consistency check of the
//     index map (restore -> get is the identity on [0, ncomp), every index tuple lands in range).
#pragma once

#include <AMReX.H>

#include <concepts>
#include <type_traits>

#include "IndexArray.hpp"

namespace treesap {
namespace tensor {
namespace detail {

template <typename Derived> constexpr bool alias_is_consistent() {
    constexpr int rank = Derived::rank, dim = Derived::dim, ncomp = Derived::ncomp;
    for (int c = 0; c < ncomp; ++c)
        if (Derived::get_relative(Derived::restore_relative(c)) != c) return false;
    if constexpr (rank == 0) {
        return ncomp == 1 && Derived::get_relative(IndexArray<0>{}) == 0;
    } else {
        int total = 1;
        for (int r = 0; r < rank; ++r) total *= dim;
        for (int flat = 0; flat < total; ++flat) { // enumerate [0, dim)^rank by mixed-radix digits
            IndexArray<rank> idx{};
            int rem = flat;
            for (int r = 0; r < rank; ++r) {
                idx[r] = rem % dim;
                rem /= dim;
            }
            const int c = Derived::get_relative(idx);
            if (c < 0 || c >= ncomp) return false;
        }
        return true;
    }
}

} // namespace detail

template <typename Derived>
concept TensorAliasImplementation =
    requires {
        typename Derived::Base;
        requires std::derived_from<Derived, typename Derived::Base>;
        typename std::integral_constant<int, Derived::ncomp>;
        typename std::integral_constant<int, Derived::rank>;
        typename std::integral_constant<int, Derived::dim>;
        typename std::integral_constant<int, Derived::next>;
        requires Derived::ncomp > 0;
        requires Derived::rank >= 0;
        requires Derived::dim > 0;
    } && requires(int comp, IndexArray<Derived::rank> ti) {
        { Derived::restore_relative(comp) } -> std::same_as<IndexArray<Derived::rank>>;
        { Derived::get_relative(ti) } -> std::same_as<int>;
    } && requires {
        typename std::integral_constant<int, Derived::get_relative(IndexArray<Derived::rank>{})>;
        typename std::integral_constant<int, Derived::restore_relative(0)[0]>;
    } && detail::alias_is_consistent<Derived>();

template <typename Derived, int comp_base_, int ncomp_, int rank_, int dim_, typename ArrayType>
struct TensorAliasBase {
    static constexpr int comp_base = comp_base_;
    static constexpr int ncomp = ncomp_;
    static constexpr int rank = rank_;
    static constexpr int dim = dim_;
    static constexpr int next = comp_base_ + ncomp_;
    static_assert(ncomp > 0 && rank >= 0 && dim > 0);

    /// Component storage being aliased (usually the RHS argument array).
    const amrex::Array4<ArrayType>& arr;

    using arr_t = ArrayType;

    /// Register copy of all aliased components of one cell, addressed by tensor indices.
    struct Temporary {
        using TemporaryArrayType = std::remove_cv_t<ArrayType>;
        TemporaryArrayType data[ncomp]{};

        AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr TemporaryArrayType& operator()(const IndexArray<rank>& ti) {
            return data[Derived::get_relative(ti)];
        }
        AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr const TemporaryArrayType&
        operator()(const IndexArray<rank>& ti) const {
            return data[Derived::get_relative(ti)];
        }
    };

    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr bool contains(int absolute_comp) {
        return absolute_comp >= comp_base && absolute_comp < comp_base + ncomp;
    }
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr int get_absolute(const IndexArray<rank>& ti) {
        return comp_base + Derived::get_relative(ti);
    }
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr IndexArray<rank> restore_absolute(int absolute_comp) {
        return Derived::restore_relative(absolute_comp - comp_base);
    }

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE ArrayType& operator()(int i, int j, int k,
                                                                   const IndexArray<rank>& ti) const {
        return arr(i, j, k, get_absolute(ti));
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE ArrayType& operator()(const amrex::IntVect& idx,
                                                                   const IndexArray<rank>& ti) const {
        return arr(idx, get_absolute(ti));
    }

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE Temporary load(int i, int j, int k) const {
        Temporary t{};
        for (int c = 0; c < ncomp; ++c) t.data[c] = arr(i, j, k, comp_base + c);
        return t;
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE Temporary load(const amrex::IntVect& idx) const {
        return load(idx[0], idx[1], idx[2]);
    }
};

} // namespace tensor
} // namespace treesap
