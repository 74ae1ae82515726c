// Test-only right-hand side that exercises the first- and third-derivative stencils of the
// public treesap API (stencil::derivative with one direction, and with three directions both
// unmixed and mixed), which none of the built-in models use. Written against the public API
// only, so the same source compiles against the reference headers (the CPU oracle) and
// against the B200 front end (the fused sm_100a stage kernels):
//   d_t u = D_x v + D_y v + a D_xxx u + b D_xyz u
//   d_t v = D_z u + c D_xxy v + c D_yz u
// The coefficients only need to keep a few steps bounded; the system is not meant to be a
// physical model. It is linear and autonomous and templated on the value type of the array, so
// it also runs in the FP32-stage RK4 form (against the reference headers T is double).
#pragma once

#include "pde-model/PDEModelConcepts.hpp"
#include "pde-model/tensor-alias/RankNAlias.hpp"
#include "util/tensor_stencil.hpp"

template <int ngrow_> struct DerivativeProbeRHS {
    static constexpr int ncomp = 2;
    static constexpr int ngrow = ngrow_;
    static_assert(ngrow >= 2, "third derivatives need ngrow >= 2");
    static constexpr bool is_affine_autonomous = true;

    struct Workspace {};

    amrex::Real a = 1e-4, b = 2e-4, c = 1e-4;

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        using namespace treesap;
        using namespace treesap::tensor;
        using namespace treesap::stencil;
        ScalarAlias<0, const T> u{{arr}};
        ScalarAlias<u.next, const T> v{{arr}};
        static_assert(v.next == ncomp);
        if constexpr (u.contains(comp)) {
            return derivative<ngrow, 0>(v, {}, idx, geom) + derivative<ngrow, 1>(v, {}, idx, geom) +
                   T(a) * derivative<ngrow, 0, 0, 0>(u, {}, idx, geom) +
                   T(b) * derivative<ngrow, 0, 1, 2>(u, {}, idx, geom);
        } else {
            return derivative<ngrow, 2>(u, {}, idx, geom) + T(c) * derivative<ngrow, 0, 0, 1>(v, {}, idx, geom) +
                   T(c) * derivative<ngrow, 1, 2>(u, {}, idx, geom);
        }
    }
};
