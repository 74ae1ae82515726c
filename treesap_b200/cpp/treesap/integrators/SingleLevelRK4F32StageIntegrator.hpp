// treesap-b200 (no reference counterpart): RK4 with FP32 stages and FP64 time level.
//
// For affine autonomous right-hand sides F(u) = L u + f0 (AffineRHSConcept) the RK4 stages
//   k_s = F(u + a_s dt k_{s-1}) = F(u) + a_s dt L k_{s-1}
// are evaluated as
//   stage 0:  k0 = F(u)              FP64 stencil of the FP64 state, stored FP32
//   stage 1:  k1 = k0 + dt/2 L k0    FP32 stencil of k0 (ghost cells: periodic images, else 0)
//   stage 2:  k2 = k0 + dt/2 L k1
//   stage 3:  k3 = k0 + dt   L k2,   u_new = u + dt/6 (k0 + 2 k1 + 2 k2 + k3) in FP64
// HBM traffic per component and step: 12 + 8 + 12 + 28 = 60 bytes (FP64 plain form: 128).
// The FP32 quantities are stage increments, whose rounding errors are O(dt) smaller than
// rounding the stage argument u + a dt k itself, which is what keeps the FP32 form within
// ~1e-7 of the FP64 path over long runs (see tests/ and bench.py for the measured error).
//
// Boundary data must not depend on time (the BC functor declares is_time_independent):
// then the increments' ghost cells outside the domain are zero and periodic directions
// wrap as usual.
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
    using typename Base::RHSType;
    using LinearRHS = decltype(linear_part_of(std::declval<const RHSType&>()));
    using FieldF = treesap_b200::DeviceField<float>;

    static_assert(requires { requires BCType::is_time_independent; },
                  "the FP32-stage form needs time-independent boundary data");

  public:
    using Tile64 = typename detail::DefaultTile<double, ngrow, ncomp>::type;
    using Tile32 = typename detail::DefaultTile<float, ngrow, ncomp>::type;

    SingleLevelRK4F32StageIntegrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr)
        : Base(std::move(model_), block_size, ctx_), k0(this->extent(), ngrow, ncomp), k1(this->extent(), ngrow, ncomp),
          k2(this->extent(), ngrow, ncomp), lin(linear_part_of(model.get_rhs())) {}

  protected:
    amrex::Real computeNewState(amrex::Real dt) override {
        using namespace treesap_b200;
        this->launches_per_step_ = 4 + 4;
        if (this->dry_run_) return dt;
        const Layout& Lu = state_old.layout();
        const Layout& Lf = k0.layout();
        int* err = ts_context_error_word(this->ctx);
        // stage 0: k0 = F(u)
        {
            StageParams<double> sp{};
            sp.in = state_old.data();
            sp.L = Lu;
            sp.geom = geom;
            sp.time = time;
            sp.err = err;
            EpiF32S0::Params ep{k0.data(), Lf};
            using Launcher = StageLauncher<Tile64, RHSType, EpiF32S0>;
            const auto shape = Launcher::shape(Lu, this->sm_count(), this->tile_rows, this->z_chunks);
            Launcher::launch(this->tensor_map(state_old.data(), Lu, TS_F64, Launcher::box_x(), Launcher::box_y(shape)),
                             sp, model.get_rhs(), ep, shape, this->stream());
        }
        fill_increment(k0);
        lin_stage<1>(k0, k1, float(0.5 * dt), dt, err);
        fill_increment(k1);
        lin_stage<2>(k1, k2, float(0.5 * dt), dt, err);
        fill_increment(k2);
        lin_stage<3>(k2, k2, float(dt), dt, err);
        return dt;
    }

  private:
    template <int S> void lin_stage(const FieldF& in, FieldF& out, float a_dt, double dt, int* err) {
        using namespace treesap_b200;
        const Layout& Lf = in.layout();
        StageParams<float> sp{};
        sp.in = in.data();
        sp.L = Lf;
        sp.geom = geom;
        sp.time = time;
        sp.err = err;
        typename EpiF32Lin<S>::Params ep{};
        ep.k_out = (S < 3) ? out.data() : nullptr;
        ep.k0 = k0.data();
        ep.k1 = k1.data();
        ep.u_in = state_old.data();
        ep.u = state_new.data();
        ep.Lf = Lf;
        ep.Lu = state_old.layout();
        ep.a_dt = a_dt;
        ep.dt = dt;
        using Launcher = StageLauncher<Tile32, LinearRHS, EpiF32Lin<S>>;
        const auto shape = Launcher::shape(Lf, this->sm_count(), this->tile_rows, this->z_chunks);
        Launcher::launch(this->tensor_map(in.data(), Lf, TS_F32, Launcher::box_x(), Launcher::box_y(shape)), sp, lin,
                         ep, shape, this->stream());
    }

    void fill_increment(FieldF& f) {
        treesap_b200::launch_ghost_fill(f.data(), f.layout(), geom, model.get_bc(), this->bc_recs_dev, time,
                                        treesap_b200::GhostMode::Homogeneous, this->sm_count(), this->stream());
    }

    FieldF k0, k1, k2;
    LinearRHS lin;
};

} // namespace treesap
