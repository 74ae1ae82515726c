// treesap-b200: symmetric rank-2 tensor alias storing the lower triangle only
// (reference pde-model/tensor-alias/SymRank2Alias.hpp:25-62). For dim 3 the components are
// {0:(0,0), 1:(1,0), 2:(1,1), 3:(2,0), 4:(2,1), 5:(2,2)}: rel = row(row+1)/2 + col with
// row = max(a, b), col = min(a, b); restore_relative returns (row, col).
#pragma once

#include "TensorAliasBase.hpp"

namespace treesap {
namespace tensor {

template <int comp_base_ = 0, int dim_ = 3, typename ArrayType = const amrex::Real>
struct SymRank2Alias : public TensorAliasBase<SymRank2Alias<comp_base_, dim_, ArrayType>, comp_base_,
                                              (dim_ * (dim_ + 1)) / 2, 2, dim_, ArrayType> {
    using Base = TensorAliasBase<SymRank2Alias<comp_base_, dim_, ArrayType>, comp_base_, (dim_ * (dim_ + 1)) / 2, 2,
                                 dim_, ArrayType>;
    using Base::dim;
    using Base::ncomp;
    using Base::next;
    using Base::rank;

    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr int get_relative(const IndexArray<2> ti) {
        const int hi = ti[0] > ti[1] ? ti[0] : ti[1];
        const int lo = ti[0] > ti[1] ? ti[1] : ti[0];
        return hi * (hi + 1) / 2 + lo;
    }
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr IndexArray<2> restore_relative(int rel) {
        int row = 0;
        while ((row + 1) * (row + 2) / 2 <= rel) ++row;
        return {row, rel - row * (row + 1) / 2};
    }
};

static_assert(TensorAliasImplementation<SymRank2Alias<0>>);

} // namespace tensor
} // namespace treesap
