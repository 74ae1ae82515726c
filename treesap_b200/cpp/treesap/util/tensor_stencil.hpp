// treesap-b200: stencils on tensor aliases (reference util/tensor_stencil.hpp:34-98):
//   stencil::derivative<ngrow, dirs...>(alias, tensor_indices, idx, geom)
// differentiates the aliased component get_absolute(tensor_indices) of alias.arr.
#pragma once

#include "../pde-model/tensor-alias/TensorAliasBase.hpp"
#include "stencil_impl.hpp"

namespace treesap {
namespace stencil {

template <int ngrow, int d0, typename AliasType>
    requires(tensor::TensorAliasImplementation<AliasType>)
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE auto derivative(const AliasType& tensor,
                                                         const tensor::IndexArray<AliasType::rank>& tensor_indices,
                                                         const amrex::IntVect& idx, const amrex::GeometryData& geom) {
    return stencil_impl::derivative_impl<ngrow, typename AliasType::Base::arr_t, d0>::eval(
        idx[0], idx[1], idx[2], AliasType::Base::get_absolute(tensor_indices), tensor.arr, geom);
}

template <int ngrow, int d0, int d1, typename AliasType>
    requires(tensor::TensorAliasImplementation<AliasType>)
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE auto derivative(const AliasType& tensor,
                                                         const tensor::IndexArray<AliasType::rank>& tensor_indices,
                                                         const amrex::IntVect& idx, const amrex::GeometryData& geom) {
    return stencil_impl::derivative_impl<ngrow, typename AliasType::Base::arr_t, d0, d1>::eval(
        idx[0], idx[1], idx[2], AliasType::Base::get_absolute(tensor_indices), tensor.arr, geom);
}

template <int ngrow, int d0, int d1, int d2, typename AliasType>
    requires(tensor::TensorAliasImplementation<AliasType>)
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE auto derivative(const AliasType& tensor,
                                                         const tensor::IndexArray<AliasType::rank>& tensor_indices,
                                                         const amrex::IntVect& idx, const amrex::GeometryData& geom) {
    return stencil_impl::derivative_impl<ngrow, typename AliasType::Base::arr_t, d0, d1, d2>::eval(
        idx[0], idx[1], idx[2], AliasType::Base::get_absolute(tensor_indices), tensor.arr, geom);
}

} // namespace stencil
} // namespace treesap
