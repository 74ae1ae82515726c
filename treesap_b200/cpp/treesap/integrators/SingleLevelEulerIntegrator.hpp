// treesap-b200: forward Euler (reference integrators/SingleLevelEulerIntegrator.hpp:28-88):
// state_new = state_old + dt F(state_old, t), one fused kernel per step.
#pragma once

#include "../SingleLevelIntegrator.hpp"

namespace treesap {

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType>
class SingleLevelEulerIntegrator : public SingleLevelIntegrator<PDEModelType> {
    using Base = SingleLevelIntegrator<PDEModelType>;
    using Base::geom;
    using Base::model;
    using Base::ncomp;
    using Base::ngrow;
    using Base::state_new;
    using Base::state_old;
    using Base::time;
    using typename Base::RHSType;

  public:
    using Tile = typename detail::DefaultTile<double, ngrow, ncomp>::type;

    SingleLevelEulerIntegrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr,
                               treesap_b200::SlabZ slab = {}, int slab_depth = 0)
        : Base(std::move(model_), block_size, ctx_, slab, slab_depth) {}

    // ---- stage-level stepping for z slabs (ZSlabDomain.hpp): one stage reading the state.
    static constexpr int kStages = 1;
    void stage_prepare(int) {}
    typename Base::Field& stage_input(int) { return state_old; }
    typename Base::FieldRef stage_ref(int) { return {state_old.data(), state_old.layout()}; }
    void stage_fill(int, amrex::Real) {
        this->fills_this_step_ = 0;
        this->FillPatch(state_old, time);
    }
    void stage_launch(int, amrex::Real dt) { computeNewState(dt); }
    void stage_finish(amrex::Real dt) {
        ++this->steps;
        time += dt;
        swap(state_old, state_new);
    }

  protected:
    amrex::Real computeNewState(amrex::Real delta_time) override {
        const auto& L = state_old.layout();
        treesap_b200::StageParams<double> sp{};
        sp.in = state_old.data();
        sp.L = L;
        sp.geom = geom;
        sp.time = time;
        sp.err = ts_context_error_word(this->ctx);
        sp.zoff = this->slab().zoff;
        treesap_b200::EpiEuler::Params ep{state_new.data(), L, delta_time};
        using Launcher = treesap_b200::StageLauncher<Tile, RHSType, treesap_b200::EpiEuler>;
        const auto shape = Launcher::shape(L, this->sm_count(), this->tile_rows, this->z_chunks);
        const CUtensorMap& tm = this->tensor_map(state_old.data(), L, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
        if (!this->dry_run_) {
            this->take_stage_fault(sp);
            this->clock_begin(1);
            Launcher::launch(tm, this->template centre_maps<Launcher>(ep, shape), sp, model.get_rhs(), ep, shape,
                             this->stream());
            this->clock_end();
        }
        this->launches_per_step_ = 1 + this->fills_this_step_;
        return delta_time;
    }
};

} // namespace treesap
