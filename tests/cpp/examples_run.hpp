// Shared model dispatch of the example-model drivers (test infrastructure): builds the
// reference's example right-hand sides (examples/01-wave-eqn/WaveEqnRHS.hpp,
// examples/02-temporaries/NonLinearRHS.hpp, compiled unchanged) or the test-only
// DerivativeProbeRHS into a PDEModel with Dirichlet or NoOp boundaries, optionally
// Kreiss-Oliger decorated, and hands it to `run(model)`:
//   example 1: WaveEqnRHS<ngrow>            (phi, u_x, u_y, u_z)
//   example 2: NonLinearRHS<ngrow>(param)   (phi, pi), gamma = param
//   example 3: DerivativeProbeRHS<ngrow>    (u, v), ngrow >= 2
// Included by oracle/ref_examples.cpp (reference integrators on the host) and by
// tests/cpp/examples_gpu.cu (B200 front end), so both sides build identical models.
#pragma once

#include "init/ConstInit.hpp"
#include "pde-model/PDEModel.hpp"
#include "pde-model/bcs/DirichletBC.hpp"
#include "pde-model/bcs/NoOpBC.hpp"
#include "pde-model/rhs-decorators/KODecorator.hpp"

#include "DerivativeProbeRHS.hpp"
#include "NonLinearRHS.hpp"
#include "WaveEqnRHS.hpp"

#include <stdexcept>
#include <string>

namespace examples_run {

/// Descriptor fields used: n, prob_lo/hi, periodic, ngrow, ko_strength, bc, bc_values, dt.
template <class Desc> amrex::Geometry geometry(const Desc& d) {
    amrex::Box dom{{0, 0, 0}, {d.n[0] - 1, d.n[1] - 1, d.n[2] - 1}};
    amrex::RealBox rb{{d.prob_lo[0], d.prob_lo[1], d.prob_lo[2]}, {d.prob_hi[0], d.prob_hi[1], d.prob_hi[2]}};
    int per[3] = {d.periodic[0], d.periodic[1], d.periodic[2]};
    return amrex::Geometry(dom, &rb, amrex::CoordSys::cartesian, per);
}

template <int nc> amrex::Vector<std::string> names() {
    amrex::Vector<std::string> v;
    for (int n = 0; n < nc; ++n) v.push_back("u" + std::to_string(n));
    return v;
}

template <class Desc, class RHS, class Run> void with_bc(const Desc& d, const RHS& rhs, Run&& run) {
    constexpr int nc = RHS::ncomp, ng = RHS::ngrow;
    using Init = treesap::ConstInit<nc>;
    if (d.bc == 1) {
        treesap::DirichletBC<nc, ng> bc{};
        for (int n = 0; n < nc; ++n) bc.boundary_values[n] = d.bc_values[n];
        run(treesap::PDEModel<RHS, Init, treesap::DirichletBC<nc, ng>>(names<nc>(), geometry(d), d.dt, rhs, Init{0.0},
                                                                       bc));
    } else {
        run(treesap::PDEModel<RHS, Init, treesap::NoOpBC<nc, ng>>(names<nc>(), geometry(d), d.dt, rhs, Init{0.0}));
    }
}

template <class Desc, class RHS, class Run> void with_ko(const Desc& d, const RHS& rhs, Run&& run) {
    if (d.ko_strength > 0.0)
        with_bc(d, treesap::KODecorator<RHS>{rhs, d.ko_strength}, run);
    else
        with_bc(d, rhs, run);
}

template <int G, class Desc, class Run> void dispatch_g(int example, const Desc& d, double param, Run&& run) {
    if (example == 1) return with_ko(d, WaveEqnRHS<G>{}, run);
    if (example == 2) return with_ko(d, NonLinearRHS<G>(param), run);
    if constexpr (G >= 2) {
        if (example == 3) return with_ko(d, DerivativeProbeRHS<G>{}, run);
    }
    throw std::invalid_argument("unknown example model or unsupported ngrow");
}

/// Components of an example model.
inline int ncomp_of(int example) { return example == 1 ? 4 : 2; }

template <class Desc, class Run> void dispatch(int example, const Desc& d, double param, Run&& run) {
    switch (d.ngrow) {
    case 1: return dispatch_g<1>(example, d, param, run);
    case 2: return dispatch_g<2>(example, d, param, run);
    case 3: return dispatch_g<3>(example, d, param, run);
    case 4: return dispatch_g<4>(example, d, param, run);
    default: throw std::invalid_argument("ngrow must be 1..4");
    }
}

} // namespace examples_run
