// treesap-b200: boundary functor that leaves ghost cells untouched (reference pde-model/bcs/NoOpBC.hpp:28-47).
// Periodic directions are still filled with periodic images by the ghost-fill kernel.
#pragma once

#include "../PDEModelConcepts.hpp"

namespace treesap {

template <int ncomp_, int ngrow_> struct NoOpBC {
    static constexpr int ncomp = ncomp_;
    static constexpr int ngrow = ngrow_;
    static constexpr bool is_time_independent = true;
    static constexpr bool is_interior_independent = true;

    AMREX_GPU_HOST_DEVICE void operator()(amrex::IntVect const&, amrex::Array4<amrex::Real> const&, int, int,
                                          amrex::GeometryData const&, amrex::Real, const amrex::BCRec*, int,
                                          int) const {}
};

static_assert(BCConcept<NoOpBC<1, 1>>);

} // namespace treesap
