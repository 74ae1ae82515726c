// treesap-b200: classical RK4 (reference integrators/SingleLevelRK4Integrator.hpp:37-166).
//
// Same registers and arithmetic as the reference: init (= state_old), acc (= state_new),
// arg, arg_next; a = {0, 1/2, 1/2, 1} dt, b = {1/6, 1/3, 1/3, 1/6} dt computed on the host;
// stage s: k = F(input, t + a_s dt) with input = init (s = 0) or arg (s > 0, after
// swap(arg_next, arg) and a ghost fill at t + a_s dt); acc = init + b k (s = 0) or
// acc += b k; arg_next = init + a_{s+1} k (s < 3). Each stage is ONE fused kernel
// (engine/stage_kernel.cuh); each ghost fill one kernel (engine/grid_kernels.cuh).
#pragma once

#include "../SingleLevelIntegrator.hpp"

namespace treesap {

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType>
class SingleLevelRK4Integrator : public SingleLevelIntegrator<PDEModelType> {
    using Base = SingleLevelIntegrator<PDEModelType>;
    using Base::FillPatch;
    using Base::geom;
    using Base::model;
    using Base::ncomp;
    using Base::ngrow;
    using Base::state_new;
    using Base::state_old;
    using Base::steps;
    using Base::time;
    using typename Base::Field;
    using typename Base::RHSType;

  public:
    using Tile = typename detail::DefaultTile<double, ngrow, ncomp>::type;

    SingleLevelRK4Integrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr,
                             treesap_b200::SlabZ slab = {}, int slab_depth = 0)
        : Base(std::move(model_), block_size, ctx_, slab, slab_depth), arg(this->extent(), ngrow, ncomp),
          arg_next(this->extent(), ngrow, ncomp) {}

  private:
    static constexpr int stage_count = 4;
    static constexpr double a_fraction[stage_count] = {0.0, 0.5, 0.5, 1.0};
    static constexpr double b_fraction[stage_count] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

  public:
    amrex::Real computeNewState(amrex::Real delta_time) override {
        run_stage<0>(delta_time);
        run_stage<1>(delta_time);
        run_stage<2>(delta_time);
        run_stage<3>(delta_time);
        this->launches_per_step_ = 4 + this->fills_this_step_; // 4 stages + the ghost fills enqueued
        return delta_time;
    }

    // ---- stage-level stepping, for domains split into z slabs (ZSlabDomain.hpp): every slab
    // takes stage s's register step, then every slab its ghost fill (whose halo hook reads the
    // neighbours' stage-s input), then every slab its stage kernel.
    static constexpr int kStages = stage_count;
    /// Stage s > 0: the register swap that makes the previous stage's output the stage input.
    void stage_prepare(int s) {
        if (s > 0) swap(arg_next, arg);
    }
    /// The field stage s reads (valid after stage_prepare(s)).
    Field& stage_input(int s) { return s == 0 ? state_old : arg; }
    typename Base::FieldRef stage_ref(int s) { return {stage_input(s).data(), stage_input(s).layout()}; }
    /// Ghost fill (with the halo hook) of stage s's input at the stage time.
    void stage_fill(int s, amrex::Real dt) {
        if (s == 0) this->fills_this_step_ = 0;
        FillPatch(stage_input(s), time + dt * a_fraction[s]);
    }
    /// The fused stage kernel of stage s.
    void stage_launch(int s, amrex::Real dt) {
        switch (s) {
        case 0: launch_stage<0>(dt); break;
        case 1: launch_stage<1>(dt); break;
        case 2: launch_stage<2>(dt); break;
        default: launch_stage<3>(dt); break;
        }
    }
    /// After stage 3: the step's bookkeeping (counters, state swap).
    void stage_finish(amrex::Real dt) {
        this->launches_per_step_ = 4 + this->fills_this_step_;
        ++steps;
        time += dt;
        swap(state_old, state_new);
    }

  private:
    template <int s> void run_stage(amrex::Real dt) {
        if constexpr (s > 0) {
            stage_prepare(s);
            FillPatch(arg, time + dt * a_fraction[s]);
        }
        launch_stage<s>(dt);
    }

    template <int s> void launch_stage(amrex::Real dt) {
        const double a_next = dt * a_fraction[(s + 1) % stage_count];
        const double time_arg = time + dt * a_fraction[s];
        const double b = dt * b_fraction[s];
        const Field& input = (s == 0) ? state_old : arg;
        const auto& L = input.layout();
        treesap_b200::StageParams<double> sp{};
        sp.in = input.data();
        sp.L = L;
        sp.geom = geom;
        sp.time = time_arg;
        sp.err = ts_context_error_word(this->ctx);
        sp.zoff = this->slab().zoff;
        typename treesap_b200::EpiRK4<s>::Params ep{state_new.data(), arg_next.data(), state_old.data(), L, b, a_next};
        using Launcher = treesap_b200::StageLauncher<Tile, RHSType, treesap_b200::EpiRK4<s>>;
        const auto shape = Launcher::shape(L, this->sm_count(), this->tile_rows, this->z_chunks);
        const CUtensorMap& tm = this->tensor_map(input.data(), L, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
        if (this->dry_run_) return;
        const treesap_b200::CentreMaps cm = this->template centre_maps<Launcher>(ep, shape);
        this->take_stage_fault(sp);
        this->clock_begin(1 + s);
        Launcher::launch(tm, cm, sp, model.get_rhs(), ep, shape, this->stream());
        this->clock_end();
    }

    Field arg;
    Field arg_next;
};

} // namespace treesap
