// treesap-b200: PDE model with an absorbing boundary layer (reference pde-model/ABLPDEModel.hpp:29-51):
// decorates the (undecorated) RHS with ABLDecorator and forces DirichletBC(target_values).
#pragma once

#include "../init/ConstInit.hpp"
#include "PDEModel.hpp"
#include "bcs/DirichletBC.hpp"
#include "rhs-decorators/ABLDecorator.hpp"
#include "rhs-decorators/NoOpRHS.hpp"

namespace treesap {

template <typename RHSType, typename InitType, typename ABLProfileType>
class ABLPDEModel
    : public PDEModel<ABLDecorator<RHSType, ABLProfileType>, InitType, DirichletBC<RHSType::ncomp, RHSType::ngrow>> {
    using DecoratedRHSType = ABLDecorator<RHSType, ABLProfileType>;
    using BCType = DirichletBC<RHSType::ncomp, RHSType::ngrow>;
    using Base = PDEModel<DecoratedRHSType, InitType, BCType>;

  public:
    ABLPDEModel(amrex::Vector<std::string> comp_names, amrex::Geometry geom, amrex::Real dt, RHSType rhs,
                typename DecoratedRHSType::ABLData abl_data, InitType init)
        : Base(std::move(comp_names), geom, dt, DecoratedRHSType{std::move(rhs), geom, abl_data}, std::move(init),
               BCType{abl_data.target_values}) {}
};

static_assert(
    PDEModelConcept<ABLPDEModel<NoOpRHS<1, 1>, ConstInit<1>, decltype([](amrex::Real x) constexpr { return x; })>>);

} // namespace treesap
