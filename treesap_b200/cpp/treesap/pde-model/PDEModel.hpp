// treesap-b200: container of the functors and data that define a PDE model
// (reference pde-model/PDEModel.hpp:34-134). Same constructor, getters and defaults:
// BC defaults to NoOpBC, bc_recs to int_dir on every face of every component.
#pragma once

#include <AMReX.H>

#include "../init/ConstInit.hpp"
#include "PDEModelConcepts.hpp"
#include "bcs/NoOpBC.hpp"
#include "rhs-decorators/NoOpRHS.hpp"

namespace treesap {

template <typename RHSType, typename InitType, typename BCType = NoOpBC<RHSType::ncomp, RHSType::ngrow>>
    requires RHSConcept<RHSType> && BCConcept<BCType> && InitConcept<InitType>
class PDEModel {
  public:
    static constexpr int ncomp = RHSType::ncomp;
    static constexpr int ngrow = RHSType::ngrow;
    using rhs_t = RHSType;
    using init_t = InitType;
    using bc_t = BCType;

    static_assert(InitType::ncomp == ncomp, "init functor has the wrong number of components");
    static_assert(BCType::ncomp == ncomp, "BC functor has the wrong number of components");
    static_assert(BCType::ngrow == ngrow, "BC functor has the wrong ghost width");

    PDEModel(amrex::Vector<std::string> comp_names, amrex::Geometry geom, amrex::Real dt, RHSType rhs, InitType init,
             BCType bc = BCType{},
             amrex::Vector<amrex::BCRec> bc_recs = amrex::Vector<amrex::BCRec>(
                 ncomp, amrex::BCRec(AMREX_D_DECL(amrex::BCType::int_dir, amrex::BCType::int_dir, amrex::BCType::int_dir),
                                     AMREX_D_DECL(amrex::BCType::int_dir, amrex::BCType::int_dir,
                                                  amrex::BCType::int_dir))))
        : rhs(std::move(rhs)), init(std::move(init)), bc(std::move(bc)), bc_recs(std::move(bc_recs)),
          geom(std::move(geom)), comp_names(std::move(comp_names)), dt(dt) {}

    const RHSType& get_rhs() const { return rhs; }
    const InitType& get_init() const { return init; }
    const BCType& get_bc() const { return bc; }
    const amrex::Vector<amrex::BCRec>& get_bc_recs() const { return bc_recs; }
    const amrex::Geometry& get_geometry() const { return geom; }
    const amrex::Vector<std::string>& get_comp_names() const { return comp_names; }
    /// Fixed-step integrators (Euler, RK4) use this as the step width.
    amrex::Real dt_hint() const { return dt; }

  protected:
    RHSType rhs;
    InitType init;
    BCType bc;
    amrex::Vector<amrex::BCRec> bc_recs;
    amrex::Geometry geom;
    amrex::Vector<std::string> comp_names;
    amrex::Real dt;
};

static_assert(PDEModelConcept<PDEModel<NoOpRHS<1, 1>, ConstInit<1>>>);

} // namespace treesap
