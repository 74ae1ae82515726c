// Built-in tensorial wave system (12 components), a treesap user model like WaveRHS.hpp.
//
//   h_ij : SymRank2Alias<0>  (components 0..5, lower-triangular order (0,0),(1,0),(1,1),(2,0),(2,1),(2,2))
//   p_ij : SymRank2Alias<6>  (components 6..11)
//
//   d_t h_ij = p_ij
//   d_t p_ij = Lap h_ij - 1/3 delta_ij Lap(h^k_k) + 1/2 (d_i d_k h_kj + d_j d_k h_ki)
//
// In Fourier space -L is symmetric positive semi-definite on symmetric matrices
// (|k|^2 (|h|^2 - tr(h)^2/3) + |h k|^2 >= 0), and the centred discretisation keeps that
// property (D2 symbol >= D1^2 symbol), so the system is energy-stable.
#pragma once

#include "pde-model/PDEModelConcepts.hpp"
#include "pde-model/tensor-alias/SymRank2Alias.hpp"
#include "util/named_tensors.hpp"
#include "util/tensor_operations.hpp"
#include "util/tensor_stencil.hpp"

namespace tsb {

template <int ngrow_> struct TensorWaveRHS {
    static constexpr int ncomp = 12;
    static constexpr int ngrow = ngrow_;
    /// Linear in the state and independent of time (eligible for the FP32-stage RK4 form).
    static constexpr bool is_affine_autonomous = true;

    struct Workspace {};

    template <int comp, typename T>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T operator()(const amrex::IntVect idx, amrex::Real /*time*/,
                                                          const amrex::Array4<const T>& arr,
                                                          const amrex::GeometryData& geom, Workspace&) const {
        using namespace treesap;
        using namespace treesap::tensor;
        using namespace treesap::stencil;

        SymRank2Alias<0, 3, const T> h{{arr}};
        SymRank2Alias<h.next, 3, const T> p{{arr}};
        static_assert(p.next == ncomp);

        if constexpr (h.contains(comp)) {
            constexpr auto ij = h.restore_absolute(comp);
            return p(idx, ij);
        } else {
            constexpr auto ij = p.restore_absolute(comp);
            constexpr int i = ij[0];
            constexpr int j = ij[1];

            T lap = contract([&]<int a>() { return derivative<ngrow, a, a>(h, {i, j}, idx, geom); });
            T div_i = contract([&]<int k>() { return derivative<ngrow, i, k>(h, {k, j}, idx, geom); });
            T div_j = contract([&]<int k>() { return derivative<ngrow, j, k>(h, {k, i}, idx, geom); });
            T result = lap + T(0.5) * (div_i + div_j);
            if constexpr (i == j) {
                T lap_trace = contract<2>(
                    [&]<int a, int k>() { return derivative<ngrow, a, a>(h, {k, k}, idx, geom); });
                result -= T(1.0 / 3.0) * lap_trace;
            }
            return result;
        }
    }
};

} // namespace tsb
