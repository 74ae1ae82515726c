// treesap-b200: fixed-size tensor index tuple, usable in constant expressions and on the
// device (reference pde-model/tensor-alias/IndexArray.hpp:21-30).
#pragma once

#include <AMReX.H>

namespace treesap {
namespace tensor {

template <int rank_> struct IndexArray {
    static_assert(rank_ >= 0, "IndexArray rank must be non-negative");
    int data[rank_ > 0 ? rank_ : 1]{};

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr int& operator[](int i) { return data[i]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr const int& operator[](int i) const { return data[i]; }
};

} // namespace tensor
} // namespace treesap
