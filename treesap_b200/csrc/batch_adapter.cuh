// treesap-b200 C ABI: type-erased adapter from ts_batch to treesap::BatchedRK4Integrator, and
// the batch builder for the built-in scalar wave model.
#pragma once

#include <utility>
#include <vector>

#include "integrator_adapter.cuh"
#include "integrators/BatchedRK4Integrator.hpp"

namespace treesap_b200 {

struct BatchIface {
    virtual ~BatchIface() = default;
    virtual int size() const = 0;
    virtual void initialise(int instance) = 0; // from the instance's parameter table
    virtual void set_state(int instance, const double* src, bool dev) = 0;
    virtual void get_state(int instance, double* dst, bool dev) = 0;
    virtual void step(int nsteps) = 0;
    virtual void use_graph(bool enable) = 0;
    virtual void set_launch_shape(int rows, int zchunk) = 0;
    virtual std::pair<int, int> autotune(int trial_steps) = 0;
    virtual std::pair<double, long long> last_step_timing() const = 0;
    virtual cudaStream_t stream() const = 0;
};

template <class B> class BatchAdapter final : public BatchIface {
  public:
    template <class Models> BatchAdapter(ts_context* ctx, Models&& models) : b_(std::forward<Models>(models), ctx) {}
    int size() const override { return b_.size(); }
    void initialise(int i) override { b_.initialise(i); }
    void set_state(int i, const double* src, bool dev) override { b_.set_state(i, src, dev); }
    void get_state(int i, double* dst, bool dev) override { b_.get_state(i, dst, dev); }
    void step(int n) override { b_.step(n); }
    void use_graph(bool e) override { b_.use_graph(e); }
    void set_launch_shape(int r, int z) override { b_.set_launch_shape(r, z); }
    std::pair<int, int> autotune(int t) override { return b_.autotune(t); }
    std::pair<double, long long> last_step_timing() const override { return b_.last_step_timing(); }
    cudaStream_t stream() const override { return b_.stream(); }

  private:
    B b_;
};

/// Capacity (doubles) of one instance's initial-condition table: kind, count, 64 items of 6.
constexpr std::size_t kBatchTableCap = 2 + 6 * 64;

/// Batch of PDEModel<WaveRHS<G> (KO-decorated when ko_strength > 0), TableInit, DirichletBC>
/// (boundary values 0 for TS_BC_NOOP: ghost cells start at zero and are never written otherwise).
template <class RHS>
BatchIface* make_batch_for_rhs(ts_context* ctx, const ts_wave_desc* d, int count, double* tables) {
    constexpr int NC = RHS::ncomp, G = RHS::ngrow;
    using Init = TableInit<NC>;
    using BC = treesap::DirichletBC<NC, G>;
    auto build = [&](auto make_rhs) -> BatchIface* {
        using R = decltype(make_rhs(0));
        using M = treesap::PDEModel<R, Init, BC>;
        std::vector<M> models;
        models.reserve(count);
        for (int i = 0; i < count; ++i) {
            BC bc{};
            for (int c = 0; c < NC; ++c) bc.boundary_values[c] = d[i].bc == TS_BC_DIRICHLET ? d[i].bc_values[c] : 0.0;
            models.emplace_back(comp_names<NC>(), geometry_of(d[i]), d[i].dt, make_rhs(i),
                                Init{tables + i * kBatchTableCap}, bc);
        }
        if (d[0].precision == TS_PRECISION_F32_STAGE)
            return new BatchAdapter<treesap::BatchedRK4Integrator<M, true>>(ctx, std::move(models));
        return new BatchAdapter<treesap::BatchedRK4Integrator<M, false>>(ctx, std::move(models));
    };
    if (d[0].ko_strength > 0.0)
        return build([&](int i) { return treesap::KODecorator<RHS>{RHS{}, d[i].ko_strength}; });
    return build([](int) { return RHS{}; });
}

BatchIface* make_batch_g2(ts_context*, const ts_wave_desc*, int, double* tables);
BatchIface* make_batch_g4(ts_context*, const ts_wave_desc*, int, double* tables);

} // namespace treesap_b200
