// treesap-b200: constant Dirichlet boundary values (reference pde-model/bcs/DirichletBC.hpp:27-66).
// Called by the ghost-fill kernel for every ghost cell outside the domain (grown in the
// periodic directions); writes boundary_values[c] to every component of that cell,
// regardless of dcomp / numcomp, as the reference does.
#pragma once

#include "../PDEModelConcepts.hpp"

namespace treesap {

template <int ncomp_, int ngrow_> struct DirichletBC {
    static constexpr int ncomp = ncomp_;
    static constexpr int ngrow = ngrow_;
    /// The boundary data do not depend on time (lets the FP32-stage form treat stage increments as homogeneous).
    static constexpr bool is_time_independent = true;
    /// ... nor on the valid cells (lets the integrators fill static ghost cells once per buffer).
    static constexpr bool is_interior_independent = true;

    amrex::GpuArray<amrex::Real, ncomp> boundary_values{};

    AMREX_GPU_HOST_DEVICE void operator()(amrex::IntVect const& iv, amrex::Array4<amrex::Real> const& dest, int /*dcomp*/,
                                          int /*numcomp*/, amrex::GeometryData const& geom, amrex::Real /*time*/,
                                          const amrex::BCRec* /*bcr*/, int /*bcomp*/, int /*orig_comp*/) const {
        if (geom.Domain().contains(iv)) return;
        for (int c = 0; c < ncomp; ++c) dest(iv, c) = boundary_values[c];
    }
};

static_assert(BCConcept<DirichletBC<1, 1>>);

} // namespace treesap
