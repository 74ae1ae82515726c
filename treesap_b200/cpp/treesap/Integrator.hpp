// treesap-b200: integrator lifecycle (reference Integrator.hpp:48-148).
// initialise() -> initialise_impl(); step() -> pre_step(), step_impl() (returns dt),
// steps++ / time += dt, post_step(); each phase inside a ScopedTimer with the reference's names.
#pragma once

#include <AMReX.H>

#include "pde-model/PDEModelConcepts.hpp"
#include "util/PlotExporter.hpp"
#include "util/ScopedTimer.hpp"
#include "util/static_for.hpp"

namespace treesap {

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType>
class Integrator {
  protected:
    static constexpr int ncomp = PDEModelType::ncomp;
    static constexpr int ngrow = PDEModelType::ngrow;
    using RHSType = typename PDEModelType::rhs_t;
    using InitType = typename PDEModelType::init_t;
    using BCType = typename PDEModelType::bc_t;

  public:
    explicit Integrator(PDEModelType model_) : model(std::move(model_)) {}
    virtual ~Integrator() = default;

    void initialise() {
        ScopedTimer timer("Integrator::initialise()");
        initialise_impl();
    }

    void step() {
        {
            ScopedTimer timer("Integrator::step() [PRE]");
            pre_step();
        }
        {
            ScopedTimer timer("Integrator::step() [STEP]");
            const amrex::Real delta_time = step_impl();
            steps++;
            time += delta_time;
        }
        {
            ScopedTimer timer("Integrator::step() [POST]");
            post_step();
        }
    }

    /// Number of completed steps and the simulation time (treesap-b200 accessors).
    std::size_t get_steps() const { return steps; }
    amrex::Real get_time() const { return time; }
    const PDEModelType& get_model() const { return model; }

  protected:
    virtual void initialise_impl() = 0;
    virtual amrex::Real step_impl() = 0;
    virtual void pre_step() {}
    virtual void post_step() {}

    PDEModelType model;
    std::size_t steps = 0;
    amrex::Real time = 0.0;
};

} // namespace treesap
