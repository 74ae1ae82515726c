// treesap-b200: right-hand side that returns zero, for testing decorators
// (reference pde-model/rhs-decorators/NoOpRHS.hpp:19-33).
#pragma once

#include "../PDEModelConcepts.hpp"

namespace treesap {

template <int ncomp_, int ngrow_> struct NoOpRHS {
    static constexpr int ncomp = ncomp_;
    static constexpr int ngrow = ngrow_;
    static constexpr bool is_affine_autonomous = true;

    struct Workspace {};

    template <int comp, typename T = amrex::Real>
    AMREX_GPU_HOST_DEVICE T operator()(const amrex::IntVect, amrex::Real, const amrex::Array4<const T>&,
                                       const amrex::GeometryData&, Workspace&) const {
        return T(0);
    }
};

static_assert(RHSConcept<NoOpRHS<1, 1>>);

} // namespace treesap
