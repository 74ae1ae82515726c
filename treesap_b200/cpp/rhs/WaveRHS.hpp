// Built-in right-hand sides of the scalar wave family, written as ordinary treesap user
// models (RHSConcept, pde-model/PDEModelConcepts.hpp:44-64 of the reference).
//
// The same source compiles against the reference headers (the CPU oracle) and against the
// B200 front end of this package, which is what makes it a parity fixture: one user model,
// two frameworks. Only the public treesap API is used (aliases, stencil::derivative,
// tensor::contract), in the style of the reference's examples/01-wave-eqn/WaveEqnRHS.hpp.
//
// Every operator() is templated on the value type T of the array it reads, so the front
// end can evaluate the model on FP32 stage arrays; against the reference (which passes
// Array4<const amrex::Real>) T is deduced as double.
#pragma once

#include "pde-model/PDEModelConcepts.hpp"
#include "pde-model/tensor-alias/RankNAlias.hpp"
#include "util/tensor_operations.hpp"
#include "util/tensor_stencil.hpp"

namespace tsb {

/// Wave speed c(x) = 1 everywhere.
struct UnitSpeed {
    template <typename T> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T c2(const amrex::IntVect&) const { return T(1); }
};

/// Wave speed squared c(x)^2 read from a cell-centred field without ghost cells
/// (x fastest, row pitch `jstride`, plane pitch `kstride`, index origin at the domain's
/// small end). The field is only read at the stencil centre.
template <typename S> struct FieldSpeed {
    const S* c2_data;
    long long jstride, kstride;
    template <typename T> AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T c2(const amrex::IntVect& iv) const {
        return T(c2_data[iv[0] + iv[1] * jstride + iv[2] * kstride]);
    }
};

/**
 * First-order-in-time scalar wave system, components {phi, pi}:
 *   d_t phi = pi,
 *   d_t pi  = c(x)^2 * sum_a D2_aa phi        (centred stencils of half-width ngrow).
 */
template <int ngrow_, typename Speed = UnitSpeed> struct WaveRHS {
    static constexpr int ncomp = 2;
    static constexpr int ngrow = ngrow_;
    /// Linear in the state and independent of time (eligible for the FP32-stage RK4 form).
    static constexpr bool is_affine_autonomous = true;

    struct Workspace {};

    Speed speed{};

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real /*time*/,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        using namespace treesap;
        using namespace treesap::tensor;
        using namespace treesap::stencil;

        ScalarAlias<0, const T> phi{{arr}};
        ScalarAlias<phi.next, const T> pi{{arr}};
        static_assert(pi.next == ncomp);

        if constexpr (phi.contains(comp)) {
            return pi(idx, {});
        } else {
            T laplacian = contract([&]<int a>() { return derivative<ngrow, a, a>(phi, {}, idx, geom); });
            return speed.template c2<T>(idx) * laplacian;
        }
    }
};

} // namespace tsb
