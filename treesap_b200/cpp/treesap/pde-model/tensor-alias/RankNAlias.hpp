// treesap-b200: dense rank-N tensor alias (reference pde-model/tensor-alias/RankNAlias.hpp:27-106).
// Component map: little-endian mixed radix, rel = sum_i dim^i * index_i.
#pragma once

#include "../../util/cexprmath.hpp"
#include "TensorAliasBase.hpp"

namespace treesap {
namespace tensor {

template <int comp_base_, int rank_, int dim_ = 3, typename ArrayType = const amrex::Real>
struct RankNAlias : public TensorAliasBase<RankNAlias<comp_base_, rank_, dim_, ArrayType>, comp_base_,
                                           int(cexprmath::power(dim_, rank_)), rank_, dim_, ArrayType> {
    using Base = TensorAliasBase<RankNAlias<comp_base_, rank_, dim_, ArrayType>, comp_base_,
                                 int(cexprmath::power(dim_, rank_)), rank_, dim_, ArrayType>;
    using Base::dim;
    using Base::ncomp;
    using Base::next;
    using Base::rank;

    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr int get_relative(const IndexArray<rank_> ti) {
        int rel = 0;
        for (int r = rank_ - 1; r >= 0; --r) rel = rel * dim_ + ti[r];
        return rel;
    }
    static AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr IndexArray<rank_> restore_relative(int rel) {
        IndexArray<rank_> ti{};
        for (int r = 0; r < rank_; ++r) {
            ti[r] = rel % dim_;
            rel /= dim_;
        }
        return ti;
    }
};

template <int comp_base_ = 0, typename ArrayType = const amrex::Real, int dim_ = 3>
using ScalarAlias = RankNAlias<comp_base_, 0, dim_, ArrayType>;
template <int comp_base_ = 0, typename ArrayType = const amrex::Real, int dim_ = 3>
using VectorAlias = RankNAlias<comp_base_, 1, dim_, ArrayType>;
template <int comp_base_ = 0, typename ArrayType = const amrex::Real, int dim_ = 3>
using Rank2Alias = RankNAlias<comp_base_, 2, dim_, ArrayType>;
template <int comp_base_ = 0, typename ArrayType = const amrex::Real, int dim_ = 3>
using Rank3Alias = RankNAlias<comp_base_, 3, dim_, ArrayType>;
template <int comp_base_ = 0, typename ArrayType = const amrex::Real, int dim_ = 3>
using Rank4Alias = RankNAlias<comp_base_, 4, dim_, ArrayType>;

static_assert(TensorAliasImplementation<ScalarAlias<0>>);
static_assert(TensorAliasImplementation<VectorAlias<0>>);
static_assert(TensorAliasImplementation<Rank2Alias<0>>);
static_assert(TensorAliasImplementation<Rank3Alias<0>>);
static_assert(TensorAliasImplementation<Rank4Alias<0>>);
static_assert(TensorAliasImplementation<RankNAlias<0, 5>>);

} // namespace tensor
} // namespace treesap
