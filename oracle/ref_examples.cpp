// ORACLE build only: the reference's example models (examples/01-wave-eqn/WaveEqnRHS.hpp and
// examples/02-temporaries/NonLinearRHS.hpp, compiled unchanged) and the test-only
// DerivativeProbeRHS, stepped by the reference's own integrators
// (integrators/SingleLevelRK4Integrator.hpp, SingleLevelEulerIntegrator.hpp) against the host
// AMReX-API shim. The state is seeded and read through configureExporter() (ref_capture.hpp).
#include "ref_fixups.hpp"

#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"

#include "examples_run.hpp"
#include "ref_capture.hpp"

#include <exception>

using namespace tsref_capture;

/// Advances state_in (valid cells, [comp][z][y][x]) by nsteps steps of example model
/// `example` (see examples_run.hpp); d->integrator selects RK4 or Euler, d->block the
/// block_size. Returns 0, or 2 on an error.
extern "C" int tsref_example_run(int example, const tsref_desc* d, double param, const double* state_in, int nsteps,
                                 double* state_out) {
    if (!d || !state_in || !state_out || nsteps < 0) return 1;
    Capture cap;
    cap.d = d;
    cap.state_in = state_in;
    cap.state_out = state_out;
    cap.nsteps = nsteps;
    cap.ncomp = examples_run::ncomp_of(example);
    try {
        examples_run::dispatch(example, *d, param, [&](auto model) {
            using M = decltype(model);
            if (d->integrator == TSREF_RK4) {
                treesap::SingleLevelRK4Integrator<M> integ(std::move(model), block_of(*d));
                drive(integ, cap);
            } else {
                treesap::SingleLevelEulerIntegrator<M> integ(std::move(model), block_of(*d));
                drive(integ, cap);
            }
        });
    } catch (const std::exception&) {
        return 2;
    }
    return 0;
}
