// treesap-b200: Kreiss-Oliger dissipation decorator (reference pde-model/rhs-decorators/KODecorator.hpp:32-74).
//   F -> F + strength * (D_KO^x + D_KO^y + D_KO^z) arr(., comp),   order defaults to ngrow.
// Models of at most kOnePassMaxComponents (4) components sum the three directions in one
// reassociated pass (stencil::kreiss_oliger_added), which differs from the reference's
// direction-by-direction sum only by rounding and issues fewer instructions. Models of more
// components sum direction by direction, as the reference does: their kernels are bound by
// register spills, and the one-pass form keeps more partial sums live (measured on the
// 12-component tensor model: FP64 stages 20% slower with the one-pass form). The threshold is
// a fixed property of the model, not of the kernel's tiling, so no tile setting changes the
// arithmetic.
// Aggregate {rhs, strength} like the reference. The operator is templated on the value type
// of the array so the same decorator runs in the FP32 stage form.
#pragma once

#include "../../util/stencil.hpp"
#include "../PDEModelConcepts.hpp"
#include "NoOpRHS.hpp"

namespace treesap {

inline constexpr int kOnePassMaxComponents = 4;

template <typename RHSType, int order_ = RHSType::ngrow>
    requires RHSConcept<RHSType>
struct KODecorator {
    static constexpr int ncomp = RHSType::ncomp;
    static constexpr int ngrow = RHSType::ngrow;
    static constexpr int order = order_;
    static_assert(order > 0 && order <= ngrow, "KO order must be in [1, ngrow]");
    static constexpr bool is_affine_autonomous = is_affine_autonomous_v<RHSType>;

    using Workspace = typename RHSType::Workspace;

    template <int comp, typename T = amrex::Real>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real time,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace& ws) const {
        if constexpr (ncomp <= kOnePassMaxComponents) {
            // F + strength (KO_x + KO_y + KO_z), all three directions in one reassociated pass
            return stencil::kreiss_oliger_added<order>(T(rhs.template operator()<comp>(idx, time, arr, geom, ws)),
                                                       arr, comp, idx, geom, strength);
        } else {
            using namespace stencil;
            T ko = kreiss_oliger<order, dir::x>(arr, comp, idx, geom);
            ko += kreiss_oliger<order, dir::y>(arr, comp, idx, geom);
            ko += kreiss_oliger<order, dir::z>(arr, comp, idx, geom);
            return T(rhs.template operator()<comp>(idx, time, arr, geom, ws)) + T(strength) * ko;
        }
    }

    /// The decorator is linear, so its linear part decorates the inner linear part.
    KODecorator linear_part() const
        requires is_affine_autonomous
    {
        return KODecorator{linear_part_of(rhs), strength};
    }

    RHSType rhs;
    amrex::Real strength;
};

static_assert(RHSConcept<KODecorator<NoOpRHS<1, 1>>>);

} // namespace treesap
