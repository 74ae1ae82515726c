// ORACLE build only: drives the reference's OWN integrators (compiled unchanged from the
// reference sources against oracle/amrex_host/) through its public API:
//   PDEModel / ABLPDEModel (pde-model/PDEModel.hpp:70-77, ABLPDEModel.hpp:47-50),
//   KODecorator{rhs, strength} (rhs-decorators/KODecorator.hpp:32-74),
//   SingleLevelRK4Integrator / SingleLevelEulerIntegrator (model, block_size),
//   initialise(), configureExporter(), step()  (Integrator.hpp:75-106, SingleLevelIntegrator.hpp:64-66).
// The state is read and seeded through configureExporter(): PlotExporter hands state_old to
// amrex::WriteSingleLevelPlotfile at the start of every pre_step (PlotExporter.hpp:54-59),
// where the shim calls the hook installed below.
#include "ref_fixups.hpp"

#include "init/ConstInit.hpp"
#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "pde-model/ABLPDEModel.hpp"
#include "pde-model/PDEModel.hpp"
#include "pde-model/bcs/DirichletBC.hpp"
#include "pde-model/bcs/NoOpBC.hpp"
#include "pde-model/rhs-decorators/KODecorator.hpp"

#include "InitFunctors.hpp"
#include "TensorWaveRHS.hpp"
#include "WaveRHS.hpp"

#include "tsref.h"

#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>

#include "ref_capture.hpp"

namespace {

using namespace tsref_capture;

template <class Model> double run_model(Model model, const tsref_desc& d, Capture& cap) {
    if (d.integrator == TSREF_RK4) {
        treesap::SingleLevelRK4Integrator<Model> integ(std::move(model), block_of(d));
        return drive(integ, cap);
    }
    treesap::SingleLevelEulerIntegrator<Model> integ(std::move(model), block_of(d));
    return drive(integ, cap);
}

// Builds PDEModel / ABLPDEModel around an undecorated RHS, optionally KO-decorated.
template <class RHS, class Init> double run_rhs(RHS rhs, Init init, const tsref_desc& d, Capture& cap) {
    constexpr int nc = RHS::ncomp, ng = RHS::ngrow;
    amrex::Geometry geom = make_geom(d);
    auto with_rhs = [&](auto r) -> double {
        using R = decltype(r);
        if (d.abl_thickness > 0) {
            amrex::GpuArray<amrex::Real, nc> target{};
            for (int n = 0; n < nc; ++n) target[n] = d.bc_values[n];
            auto run_profile = [&](auto profile) -> double {
                using P = decltype(profile);
                using M = treesap::ABLPDEModel<R, Init, P>;
                typename treesap::ABLDecorator<R, P>::ABLData abl(target, d.abl_thickness, d.abl_max_strength,
                                                                  profile);
                return run_model(M(names<nc>(), geom, d.dt, r, abl, init), d, cap);
            };
            if (d.abl_profile == 1) return run_profile(tsb::LinearProfile{});
            return run_profile(tsb::QuadraticProfile{});
        }
        if (d.bc == TSREF_BC_DIRICHLET) {
            treesap::DirichletBC<nc, ng> bc{};
            for (int n = 0; n < nc; ++n) bc.boundary_values[n] = d.bc_values[n];
            return run_model(treesap::PDEModel<R, Init, treesap::DirichletBC<nc, ng>>(names<nc>(), geom, d.dt, r,
                                                                                     init, bc),
                             d, cap);
        }
        return run_model(treesap::PDEModel<R, Init, treesap::NoOpBC<nc, ng>>(names<nc>(), geom, d.dt, r, init), d,
                         cap);
    };
    if (d.ko_strength > 0.0) return with_rhs(treesap::KODecorator<RHS>{rhs, d.ko_strength});
    return with_rhs(rhs);
}

template <int ncomp> tsb::GaussianSumInit<ncomp> gaussian_init(int n, const double* it) {
    tsb::GaussianSumInit<ncomp> g{};
    if (n > g.max_pulses) throw std::invalid_argument("too many pulses");
    g.npulses = n;
    for (int p = 0; p < n; ++p) {
        g.comp[p] = int(it[6 * p + 0]);
        g.amp[p] = it[6 * p + 1];
        g.width[p] = it[6 * p + 2];
        g.cx[p] = it[6 * p + 3];
        g.cy[p] = it[6 * p + 4];
        g.cz[p] = it[6 * p + 5];
    }
    return g;
}

template <int ncomp> tsb::FourierSumInit<ncomp> fourier_init(int n, const double* it) {
    tsb::FourierSumInit<ncomp> f{};
    if (n > f.max_modes) throw std::invalid_argument("too many modes");
    f.nmodes = n;
    for (int m = 0; m < n; ++m) {
        f.comp[m] = int(it[6 * m + 0]);
        f.amp[m] = it[6 * m + 1];
        f.kx[m] = it[6 * m + 2];
        f.ky[m] = it[6 * m + 3];
        f.kz[m] = it[6 * m + 4];
        f.phase[m] = it[6 * m + 5];
    }
    return f;
}

template <class RHS> double run_with_init(RHS rhs, const tsref_desc& d, int kind, int nitems, const double* items,
                                          Capture& cap) {
    constexpr int nc = RHS::ncomp;
    if (kind == TSREF_INIT_FOURIER) return run_rhs(rhs, fourier_init<nc>(nitems, items), d, cap);
    // TSREF_INIT_STATE seeds through the hook; the Gaussian functor with zero pulses gives 0.
    return run_rhs(rhs, gaussian_init<nc>(kind == TSREF_INIT_GAUSSIAN ? nitems : 0, items), d, cap);
}

template <int G> double dispatch_model(const tsref_desc& d, int kind, int nitems, const double* items, Capture& cap) {
    if (d.model == TSREF_MODEL_TENSOR_WAVE) return run_with_init(tsb::TensorWaveRHS<G>{}, d, kind, nitems, items, cap);
    if (d.c2) {
        tsb::WaveRHS<G, tsb::FieldSpeed<double>> rhs{};
        rhs.speed = tsb::FieldSpeed<double>{d.c2, d.n[0], (long long)d.n[0] * d.n[1]};
        return run_with_init(rhs, d, kind, nitems, items, cap);
    }
    return run_with_init(tsb::WaveRHS<G>{}, d, kind, nitems, items, cap);
}

} // namespace

#ifdef TSREF_G
// One translation unit per stencil half-width keeps the (many) template instantiations
// of the reference integrators compiling in parallel.
#define TSREF_CAT2(a, b) a##b
#define TSREF_CAT(a, b) TSREF_CAT2(a, b)
extern "C" int TSREF_CAT(tsref_run_g, TSREF_G)(const tsref_desc* d, int init_kind, int nitems, const double* items,
                                              const double* state_in, int nsteps, double* state_out, double* seconds,
                                              double* time_out) {
    Capture cap;
    cap.d = d;
    cap.state_in = (init_kind == TSREF_INIT_STATE) ? state_in : nullptr;
    cap.state_out = state_out;
    cap.nsteps = nsteps;
    cap.ncomp = (d->model == TSREF_MODEL_TENSOR_WAVE) ? 12 : 2;
    try {
        const double secs = dispatch_model<TSREF_G>(*d, init_kind, nitems, items, cap);
        if (seconds) *seconds = secs;
        if (time_out) *time_out = cap.time;
    } catch (const std::exception&) {
        return 2;
    }
    return 0;
}
#else
extern "C" {
int tsref_run_g1(const tsref_desc*, int, int, const double*, const double*, int, double*, double*, double*);
int tsref_run_g2(const tsref_desc*, int, int, const double*, const double*, int, double*, double*, double*);
int tsref_run_g3(const tsref_desc*, int, int, const double*, const double*, int, double*, double*, double*);
int tsref_run_g4(const tsref_desc*, int, int, const double*, const double*, int, double*, double*, double*);

int tsref_run(const tsref_desc* d, int init_kind, int nitems, const double* items, const double* state_in, int nsteps,
              double* state_out, double* seconds, double* time_out) {
    if (!d || !state_out || nsteps < 0) return 1;
    for (int q = 0; q < 3; ++q)
        if (d->n[q] < 1 || d->n[q] < d->ngrow) return 1;
    if (init_kind == TSREF_INIT_STATE && !state_in) return 1;
    switch (d->ngrow) {
    case 1: return tsref_run_g1(d, init_kind, nitems, items, state_in, nsteps, state_out, seconds, time_out);
    case 2: return tsref_run_g2(d, init_kind, nitems, items, state_in, nsteps, state_out, seconds, time_out);
    case 3: return tsref_run_g3(d, init_kind, nitems, items, state_in, nsteps, state_out, seconds, time_out);
    case 4: return tsref_run_g4(d, init_kind, nitems, items, state_in, nsteps, state_out, seconds, time_out);
    default: return 1;
    }
}

int tsref_threads(void) { return amrex::host_threads(); }
}
#endif
