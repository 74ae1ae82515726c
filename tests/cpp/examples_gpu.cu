// GPU side of the example-model parity tests (test infrastructure): the reference's example
// right-hand sides (compiled unchanged) and the test-only DerivativeProbeRHS, stepped by the
// B200 front end's integrators (fused sm_100a stage kernels) from a given state. Same model
// dispatch as the oracle build (examples_run.hpp); built by oracle/Makefile against
// libtreesap_b200.so.
#include <AMReX.H>

#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4F32StageIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"

#include "examples_run.hpp"
#include "tsref.h"

#include <exception>
#include <cstdio>

/// Integrator code of the front end's FP32-stage RK4 form (GPU side only; the reference has
/// no such form, so its results are compared with the reference's FP64 RK4).
constexpr int kRK4F32Stage = 2;

#ifdef TSB_EX_G
// One translation unit per stencil half-width (TSB_EX_G = 1..4), compiled in parallel.
#define TSB_EX_CAT2(a, b) a##b
#define TSB_EX_CAT(a, b) TSB_EX_CAT2(a, b)
extern "C" int TSB_EX_CAT(tsb_example_run_g, TSB_EX_G)(int example, const tsref_desc* d, double param,
                                                     const double* state_in, int nsteps, double* state_out) {
    try {
        examples_run::dispatch_g<TSB_EX_G>(example, *d, param, [&](auto model) {
            using M = decltype(model);
            const amrex::IntVect block{d->block[0] > 0 ? d->block[0] : d->n[0], d->block[1] > 0 ? d->block[1] : d->n[1],
                                       d->block[2] > 0 ? d->block[2] : d->n[2]};
            auto go = [&](auto& integ) {
                integ.set_state(state_in);
                for (int s = 0; s < nsteps; ++s) integ.step();
                integ.get_state(state_out);
            };
            if (d->integrator == TSREF_RK4) {
                treesap::SingleLevelRK4Integrator<M> integ(std::move(model), block);
                go(integ);
            } else if (d->integrator == kRK4F32Stage) {
                if constexpr (treesap::AffineRHSConcept<typename M::rhs_t>) {
                    treesap::SingleLevelRK4F32StageIntegrator<M> integ(std::move(model), block);
                    go(integ);
                } else {
                    throw std::invalid_argument("the FP32-stage form needs an affine model");
                }
            } else {
                treesap::SingleLevelEulerIntegrator<M> integ(std::move(model), block);
                go(integ);
            }
        });
    } catch (const std::exception& e) {
        std::fprintf(stderr, "tsb_example_run: %s\n", e.what());
        return 2;
    }
    return 0;
}
#else
extern "C" {
int tsb_example_run_g1(int, const tsref_desc*, double, const double*, int, double*);
int tsb_example_run_g2(int, const tsref_desc*, double, const double*, int, double*);
int tsb_example_run_g3(int, const tsref_desc*, double, const double*, int, double*);
int tsb_example_run_g4(int, const tsref_desc*, double, const double*, int, double*);

/// Same contract as tsref_example_run: state_in -> nsteps steps -> state_out (host arrays of
/// valid cells, [comp][z][y][x]). Returns 0, 1 on an invalid argument, or 2 with the message on
/// stderr.
int tsb_example_run(int example, const tsref_desc* d, double param, const double* state_in, int nsteps,
                    double* state_out) {
    if (!d || !state_in || !state_out || nsteps < 0) return 1;
    switch (d->ngrow) {
    case 1: return tsb_example_run_g1(example, d, param, state_in, nsteps, state_out);
    case 2: return tsb_example_run_g2(example, d, param, state_in, nsteps, state_out);
    case 3: return tsb_example_run_g3(example, d, param, state_in, nsteps, state_out);
    case 4: return tsb_example_run_g4(example, d, param, state_in, nsteps, state_out);
    default: return 1;
    }
}
}
#endif
