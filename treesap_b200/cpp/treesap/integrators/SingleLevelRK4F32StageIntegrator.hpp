// treesap-b200 (no reference counterpart): RK4 with FP32 stages and FP64 time level.
//
// For affine autonomous right-hand sides F(u) = L u + f0 (AffineRHSConcept) the RK4 stages
//   k_s = F(u + a_s dt k_{s-1}) = F(u) + a_s dt L k_{s-1}
// are carried as k0 plus FP32 differences d_s = k_s - k0:
//   stage 0:  k0 = F(u)                  FP64 stencil of the FP64 state, k0 stored FP64;
//             u_p = u + dt k0            written in FP64
//   stage 1:  d1 = dt/2 L k0             FP64 stencil of k0, d1 stored FP32
//   stage 2:  d2 = d1 + dt/2 L d1        FP32 stencil of d1  (d2 = dt/2 L k1)
//   stage 3:  d3 = 2 d1 + dt L d2        FP32 stencil of d2  (d3 = dt L k2)
//             u_new = u_p + dt/6 (2 d1 + 2 d2 + d3)   in FP64
// Stencils of full-magnitude fields (u, k0) run in FP64: a centred 8th-order D2 cancels
// ~1e6-fold, which FP32 arithmetic cannot resolve to the 1e-6 target over 1000 steps. The
// FP32 stencils act on the differences d_s, which are O(dt |L|) smaller than the stage values.
// HBM traffic per component and step: 24 + 12 + 8 + 24 = 68 bytes (FP64 plain form: 128).
//
// Ghost cells of k0 and of the differences: periodic images in periodic directions, zero
// elsewhere; exact when the boundary data do not depend on time (the BC functor declares
// is_time_independent), since every stage argument then has the ghost values of u.
#pragma once

#include "../SingleLevelIntegrator.hpp"

namespace treesap {

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType> && AffineRHSConcept<typename PDEModelType::rhs_t>
class SingleLevelRK4F32StageIntegrator : public SingleLevelIntegrator<PDEModelType> {
    using Base = SingleLevelIntegrator<PDEModelType>;
    using Base::FillPatch;
    using Base::geom;
    using Base::model;
    using Base::ncomp;
    using Base::ngrow;
    using Base::state_new;
    using Base::state_old;
    using Base::time;
    using typename Base::BCType;
    using typename Base::Field;
    using typename Base::RHSType;
    using LinearRHS = decltype(linear_part_of(std::declval<const RHSType&>()));
    using FieldF = treesap_b200::DeviceField<float>;

    static_assert(requires { requires BCType::is_time_independent; },
                  "the FP32-stage form needs time-independent boundary data");

  public:
    using Tile64 = typename detail::DefaultTile<double, ngrow, ncomp>::type;
    using Tile32 = typename detail::DefaultTile<float, ngrow, ncomp>::type;

    SingleLevelRK4F32StageIntegrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr,
                                     treesap_b200::SlabZ slab = {}, int slab_depth = 0)
        : Base(std::move(model_), block_size, ctx_, slab, slab_depth), k0(this->extent(), ngrow, ncomp),
          d1(this->extent(), ngrow, ncomp), d2(this->extent(), ngrow, ncomp), lin(linear_part_of(model.get_rhs())) {}

    // ---- stage-level stepping for z slabs (ZSlabDomain.hpp, ts_slab_*): the inputs of the four
    // stages are u, k0 (FP64) and d1, d2 (FP32).
    static constexpr int kStages = 4;
    void stage_prepare(int) {}
    typename Base::FieldRef stage_ref(int s) {
        switch (s) {
        case 0: return {state_old.data(), state_old.layout()};
        case 1: return {k0.data(), k0.layout()};
        case 2: return {d1.data(), d1.layout()};
        default: return {d2.data(), d2.layout()};
        }
    }
    void stage_fill(int s, amrex::Real) {
        switch (s) {
        case 0:
            this->fills_this_step_ = 0;
            this->FillPatch(state_old, time);
            break;
        case 1: fill_increment(k0); break;
        case 2: fill_increment(d1); break;
        default: fill_increment(d2); break;
        }
    }
    void stage_launch(int s, amrex::Real dt) {
        if (this->dry_run_) return;
        int* err = ts_context_error_word(this->ctx);
        switch (s) {
        case 0: launch_s0(dt, err); break;
        case 1: launch_s1(dt, err); break;
        case 2: lin_stage<2>(d1, d2, float(0.5 * dt), dt, err); break;
        default: lin_stage<3>(d2, d2, float(dt), dt, err); break;
        }
    }
    void stage_finish(amrex::Real dt) {
        this->launches_per_step_ = 4 + this->fills_this_step_;
        ++this->steps;
        time += dt;
        swap(state_old, state_new);
    }

  protected:
    amrex::Real computeNewState(amrex::Real dt) override {
        if (this->dry_run_) return dt;
        int* err = ts_context_error_word(this->ctx);
        launch_s0(dt, err);
        fill_increment(k0);
        launch_s1(dt, err);
        fill_increment(d1);
        lin_stage<2>(d1, d2, float(0.5 * dt), dt, err);
        fill_increment(d2);
        lin_stage<3>(d2, d2, float(dt), dt, err);
        this->launches_per_step_ = 4 + this->fills_this_step_;
        return dt;
    }

  private:
    /// stage 0: k0 = F(u), u_p = u + dt k0 (into state_new)
    void launch_s0(amrex::Real dt, int* err) {
        using namespace treesap_b200;
        const Layout& Lu = state_old.layout();
        {
            StageParams<double> sp{};
            sp.in = state_old.data();
            sp.L = Lu;
            sp.geom = geom;
            sp.time = time;
            sp.err = err;
            sp.zoff = this->slab().zoff;
            EpiF32S0::Params ep{k0.data(), state_new.data(), Lu, dt};
            using Launcher = StageLauncher<Tile64, RHSType, EpiF32S0>;
            const auto shape = Launcher::shape(Lu, this->sm_count(), this->tile_rows, this->z_chunks);
            const CUtensorMap& tm =
                this->tensor_map(state_old.data(), Lu, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
            const CentreMaps cm = this->template centre_maps<Launcher>(ep, shape);
            this->take_stage_fault(sp);
            this->clock_begin(1);
            Launcher::launch(tm, cm, sp, model.get_rhs(), ep, shape, this->stream());
            this->clock_end();
        }
    }
    /// stage 1: d1 = dt/2 L k0 (FP64 stencil)
    void launch_s1(amrex::Real dt, int* err) {
        using namespace treesap_b200;
        const Layout& Lu = state_old.layout();
        const Layout& Lf = d1.layout();
        {
            StageParams<double> sp{};
            sp.in = k0.data();
            sp.L = Lu;
            sp.geom = geom;
            sp.time = time;
            sp.err = err;
            sp.zoff = this->slab().zoff;
            EpiF32S1::Params ep{d1.data(), Lf, 0.5 * dt};
            using Launcher = StageLauncher<Tile64, LinearRHS, EpiF32S1>;
            const auto shape = Launcher::shape(Lu, this->sm_count(), this->tile_rows, this->z_chunks);
            const CUtensorMap& tm = this->tensor_map(k0.data(), Lu, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
            const CentreMaps cm = this->template centre_maps<Launcher>(ep, shape);
            this->take_stage_fault(sp);
            this->clock_begin(2);
            Launcher::launch(tm, cm, sp, lin, ep, shape, this->stream());
            this->clock_end();
        }
    }

    template <int S> void lin_stage(const FieldF& in, FieldF& out, float a_dt, double dt, int* err) {
        using namespace treesap_b200;
        const Layout& Lf = in.layout();
        StageParams<float> sp{};
        sp.in = in.data();
        sp.L = Lf;
        sp.geom = geom;
        sp.time = time;
        sp.err = err;
        sp.zoff = this->slab().zoff;
        typename EpiF32Lin<S>::Params ep{};
        ep.d_out = (S < 3) ? out.data() : nullptr;
        ep.d1 = d1.data();
        ep.u = state_new.data();
        ep.Lf = Lf;
        ep.Lu = state_new.layout();
        ep.a_dt = a_dt;
        ep.dt = dt;
        using Launcher = StageLauncher<Tile32, LinearRHS, EpiF32Lin<S>>;
        const auto shape = Launcher::shape(Lf, this->sm_count(), this->tile_rows, this->z_chunks);
        const CUtensorMap& tm = this->tensor_map(in.data(), Lf, TS_F32, Launcher::box_x(), Launcher::box_y(shape));
        const CentreMaps cm = this->template centre_maps<Launcher>(ep, shape);
        this->take_stage_fault(sp);
        this->clock_begin(1 + S);
        Launcher::launch(tm, cm, sp, lin, ep, shape, this->stream());
        this->clock_end();
    }

    template <class F> void fill_increment(F& f) {
        if (this->dry_run_) return;
        this->halo(f);
        if (!this->ghost_fill_needed(f.data())) return;
        this->count_fill();
        this->clock_begin(0);
        treesap_b200::launch_ghost_fill(f.data(), f.layout(), geom, model.get_bc(), this->bc_recs_dev, time,
                                        treesap_b200::GhostMode::Homogeneous, this->sm_count(), this->stream(),
                                        this->slab());
        this->clock_end();
    }

    Field k0;
    FieldF d1, d2;
    LinearRHS lin;
};

} // namespace treesap
