// treesap-b200: constant initial condition (reference init/ConstInit.hpp:19-40).
#pragma once

#include "../pde-model/PDEModelConcepts.hpp"

namespace treesap {

template <int ncomp_> struct ConstInit {
    static_assert(ncomp_ > 0, "ConstInit needs at least one component");
    static constexpr int ncomp = ncomp_;

    amrex::Real value;

    template <int comp>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real operator()(amrex::Real, amrex::Real, amrex::Real) const {
        return value;
    }
};

static_assert(InitConcept<ConstInit<1>>);

} // namespace treesap
