// ORACLE build only. Included after the reference's util/stencil.hpp and before its
// rhs-decorators/KODecorator.hpp.
//
// KODecorator::operator() (reference pde-model/rhs-decorators/KODecorator.hpp:64-66) calls
//     kreiss_oliger<order, dir>(idx, comp, arr, geom)
// while kreiss_oliger is declared as (arr, comp, idx, geom) (reference util/stencil.hpp:77-80),
// so the decorator cannot be instantiated as published. This overload accepts the argument
// order used at the call site and forwards to the published operator, leaving the reference
// files untouched. The B200 front end accepts both orders for the same reason.
#pragma once

#include "util/stencil.hpp"

namespace treesap {
namespace stencil {
template <int order, int dir, typename ArrayType>
inline ArrayType kreiss_oliger(const amrex::IntVect& idx, int comp, const amrex::Array4<ArrayType>& arr,
                               const amrex::GeometryData& geom) {
    return kreiss_oliger<order, dir, ArrayType>(arr, comp, idx, geom);
}
} // namespace stencil
} // namespace treesap
