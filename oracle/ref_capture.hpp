// ORACLE build only: capture of the reference integrators' state through their public API.
// PlotExporter hands state_old to amrex::WriteSingleLevelPlotfile at the start of every
// pre_step (PlotExporter.hpp:54-59 of the reference), where the host shim calls the hook
// installed here: step 0 seeds the initial state, step nsteps copies the result out and
// stops the run. Shared by ref_entry.cpp (built-in models) and ref_examples.cpp (the
// reference's example models).
#pragma once

#include "tsref.h"

#include <AMReX.H>

#include <chrono>
#include <string>

namespace tsref_capture {

struct StopAfterCapture {};

struct Capture {
    const tsref_desc* d = nullptr;
    const double* state_in = nullptr;
    double* state_out = nullptr;
    int nsteps = 0;
    int ncomp = 0;
    double time = 0.0;
};

template <class F> void for_valid(const tsref_desc& d, F&& f) {
    for (int k = 0; k < d.n[2]; ++k)
        for (int j = 0; j < d.n[1]; ++j)
            for (int i = 0; i < d.n[0]; ++i) f(i, j, k, (std::size_t(k) * d.n[1] + j) * d.n[0] + i);
}

inline void plot_hook(void* user, const amrex::MultiFab& mf, int step, amrex::Real time) {
    auto* c = static_cast<Capture*>(user);
    const tsref_desc& d = *c->d;
    const std::size_t ncell = std::size_t(d.n[0]) * d.n[1] * d.n[2];
    if (step == 0 && c->state_in) { // seed the initial state before the first ghost fill
        auto& m = const_cast<amrex::MultiFab&>(mf);
        for (int b = 0; b < m.size(); ++b) {
            amrex::Array4<amrex::Real> a = m.array(b);
            const amrex::Box bx = m.boxArray()[b];
            for_valid(d, [&](int i, int j, int k, std::size_t q) {
                if (!bx.contains(i, j, k)) return;
                for (int n = 0; n < c->ncomp; ++n) a(i, j, k, n) = c->state_in[n * ncell + q];
            });
        }
    }
    if (step == c->nsteps) {
        for (int b = 0; b < mf.size(); ++b) {
            amrex::Array4<const amrex::Real> a = mf.const_array(b);
            const amrex::Box bx = mf.boxArray()[b];
            for_valid(d, [&](int i, int j, int k, std::size_t q) {
                if (!bx.contains(i, j, k)) return;
                for (int n = 0; n < c->ncomp; ++n) c->state_out[n * ncell + q] = a(i, j, k, n);
            });
        }
        c->time = time;
        throw StopAfterCapture{};
    }
}

template <class Integrator> double drive(Integrator& integ, Capture& cap) {
    integ.initialise();
    integ.configureExporter("oracle-capture", 1);
    amrex::plot_hook() = &plot_hook;
    amrex::plot_hook_user() = &cap;
    auto t0 = std::chrono::steady_clock::now();
    try {
        for (int s = 0; s <= cap.nsteps; ++s) integ.step(); // the last call only captures
    } catch (const StopAfterCapture&) {
    }
    auto t1 = std::chrono::steady_clock::now();
    amrex::plot_hook() = nullptr;
    return std::chrono::duration<double>(t1 - t0).count();
}

inline amrex::Geometry make_geom(const tsref_desc& d) {
    amrex::Box dom{{0, 0, 0}, {d.n[0] - 1, d.n[1] - 1, d.n[2] - 1}};
    amrex::RealBox rb{{d.prob_lo[0], d.prob_lo[1], d.prob_lo[2]}, {d.prob_hi[0], d.prob_hi[1], d.prob_hi[2]}};
    int is_per[3] = {d.periodic[0], d.periodic[1], d.periodic[2]};
    return amrex::Geometry(dom, &rb, amrex::CoordSys::cartesian, is_per);
}

inline amrex::IntVect block_of(const tsref_desc& d) {
    return {d.block[0] > 0 ? d.block[0] : d.n[0], d.block[1] > 0 ? d.block[1] : d.n[1],
            d.block[2] > 0 ? d.block[2] : d.n[2]};
}

template <int ncomp> amrex::Vector<std::string> names() {
    amrex::Vector<std::string> v;
    for (int n = 0; n < ncomp; ++n) v.push_back("u" + std::to_string(n));
    return v;
}

} // namespace tsref_capture
