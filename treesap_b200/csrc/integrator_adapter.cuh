// treesap-b200 C ABI: type-erased adapter from ts_integrator to the header front end's
// integrators, and the model builder for the built-in models (ts_wave_desc).
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <treesap_b200.h>

#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4F32StageIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "pde-model/ABLPDEModel.hpp"
#include "pde-model/PDEModel.hpp"
#include "pde-model/bcs/DirichletBC.hpp"
#include "pde-model/bcs/NoOpBC.hpp"
#include "pde-model/rhs-decorators/KODecorator.hpp"
#include "util/expression.hpp"

#include "InitFunctors.hpp"
#include "TensorWaveRHS.hpp"
#include "WaveRHS.hpp"

namespace treesap_b200 {

/// Initial condition read from a device parameter table:
///   table[0] = kind (TS_INIT_GAUSSIAN / TS_INIT_FOURIER), table[1] = count, then 6 doubles per item
///   (Gaussian: comp, A, w, cx, cy, cz; Fourier: comp, A, kx, ky, kz, phase);
///   kind TS_INIT_EXPRESSION: table[1] = NC, table[2 + c] = start (in doubles) and
///   table[2 + NC + c] = length (instructions) of component c's postfix program
///   (treesap::expr::Instr, two doubles each), the programs after the header.
/// Same formulas and summation order as tsb::GaussianSumInit / tsb::FourierSumInit.
template <int NC> struct TableInit {
    static constexpr int ncomp = NC;
    const double* table = nullptr;

    template <int c>
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE amrex::Real operator()(amrex::Real x, amrex::Real y, amrex::Real z) const {
        const int kind = int(table[0]), n = int(table[1]);
        if (kind == TS_INIT_EXPRESSION) {
            const auto* code = reinterpret_cast<const treesap::expr::Instr*>(table + int(table[2 + c]));
            return treesap::expr::eval(code, int(table[2 + NC + c]), x, y, z);
        }
        amrex::Real v = 0.0;
        for (int p = 0; p < n; ++p) {
            const double* it = table + 2 + 6 * p;
            if (int(it[0]) != c) continue;
            if (kind == TS_INIT_GAUSSIAN) {
                const amrex::Real dx = x - it[3], dy = y - it[4], dz = z - it[5];
                v += it[1] * std::exp(-(dx * dx + dy * dy + dz * dz) / (it[2] * it[2]));
            } else {
                constexpr amrex::Real two_pi = 6.283185307179586476925286766559;
                v += it[1] * std::cos(two_pi * (it[2] * x + it[3] * y + it[4] * z) + it[5]);
            }
        }
        return v;
    }
};

struct IntegratorIface {
    virtual ~IntegratorIface() = default;
    virtual int ncomp() const = 0;
    virtual void initialise(int kind, int nitems, const double* items) = 0;
    /// Expression initial condition: one expression of x, y, z per component.
    virtual void initialise_expressions(int count, const char* const* exprs) = 0;
    virtual void set_state(const double* src, bool dev) = 0;
    virtual void get_state(double* dst, bool dev) = 0;
    virtual void step() = 0;
    virtual void step_host_only() = 0; // host bookkeeping of one step, no device work (graph replay)
    virtual double time() const = 0;
    virtual long long steps() const = 0;
    virtual void* state_ptr() = 0;
    virtual Layout state_layout() const = 0;
    virtual long long launches_per_step() const = 0;
    virtual void attach_clock(treesap::KernelClock* c) = 0;
    virtual void set_launch_shape(int rows, int chunks) = 0;
    virtual bool state_is_finite() = 0;
};

/// Exposes the protected time / step counters of the front-end integrators.
/// (The parameter table and the speed field are owned by the ts_integrator, not by the adapter.)
template <class Integ> struct Exposed : Integ {
    using Integ::Integ;
    void set_clock(double t, std::size_t s) {
        this->time = t;
        this->steps = s;
    }
};

template <class Integ, int NC> class Adapter final : public IntegratorIface {
  public:
    template <class Model>
    Adapter(ts_context* ctx, Model&& model, double* table, std::size_t table_cap)
        : integ_(std::forward<Model>(model), amrex::IntVect{1 << 30, 1 << 30, 1 << 30}, ctx), table_(table),
          table_cap_(table_cap) {}
    int ncomp() const override { return NC; }
    void initialise(int kind, int nitems, const double* items) override {
        if (nitems < 0 || std::size_t(2 + 6 * nitems) > table_cap_) throw std::invalid_argument("too many init items");
        std::vector<double> host(2 + 6 * std::size_t(nitems));
        host[0] = kind;
        host[1] = nitems;
        for (int q = 0; q < 6 * nitems; ++q) host[2 + q] = items[q];
        cuda_check(cudaMemcpyAsync(table_, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice,
                                   integ_.stream()),
                   "cudaMemcpyAsync(init table)");
        integ_.initialise();
        cuda_check(cudaStreamSynchronize(integ_.stream()), "cudaStreamSynchronize(initialise)");
    }
    void initialise_expressions(int count, const char* const* exprs) override {
        if (count != NC) throw std::invalid_argument("one expression per component is required");
        std::vector<double> host(2 + 2 * NC);
        host[0] = TS_INIT_EXPRESSION;
        host[1] = NC;
        for (int c = 0; c < NC; ++c) {
            if (!exprs[c]) throw std::invalid_argument("null expression");
            const std::vector<treesap::expr::Instr> code = treesap::expr::Compiler::compile(exprs[c]);
            host[2 + c] = double(host.size());
            host[2 + NC + c] = double(code.size());
            const std::size_t at = host.size();
            host.resize(at + 2 * code.size());
            std::memcpy(host.data() + at, code.data(), sizeof(treesap::expr::Instr) * code.size());
        }
        if (host.size() > table_cap_) throw std::invalid_argument("expressions too long for the parameter table");
        cuda_check(cudaMemcpyAsync(table_, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice,
                                   integ_.stream()),
                   "cudaMemcpyAsync(init table)");
        integ_.initialise();
        cuda_check(cudaStreamSynchronize(integ_.stream()), "cudaStreamSynchronize(initialise)");
    }
    void set_state(const double* src, bool dev) override { integ_.set_state(src, dev); }
    void get_state(double* dst, bool dev) override { integ_.get_state(dst, dev); }
    void step() override { integ_.step(); }
    void step_host_only() override { integ_.step_host_only(); }
    double time() const override { return integ_.get_time(); }
    long long steps() const override { return (long long)integ_.get_steps(); }
    void* state_ptr() override { return integ_.state().data(); }
    Layout state_layout() const override { return integ_.state().layout(); }
    long long launches_per_step() const override { return integ_.launches_per_step(); }
    void attach_clock(treesap::KernelClock* c) override { integ_.attach_clock(c); }
    void set_launch_shape(int rows, int chunks) override { integ_.set_launch_shape(rows, chunks); }
    bool state_is_finite() override { return integ_.state_is_finite(); }

  private:
    Exposed<Integ> integ_;
    double* table_;
    std::size_t table_cap_;
};

constexpr std::size_t kInitTableCap = 2 + 6 * 512;

inline amrex::Geometry geometry_of(const ts_wave_desc& d) {
    amrex::Box dom{{0, 0, 0}, {d.n[0] - 1, d.n[1] - 1, d.n[2] - 1}};
    amrex::RealBox rb{{d.prob_lo[0], d.prob_lo[1], d.prob_lo[2]}, {d.prob_hi[0], d.prob_hi[1], d.prob_hi[2]}};
    int per[3] = {d.periodic[0] != 0, d.periodic[1] != 0, d.periodic[2] != 0};
    return amrex::Geometry(dom, &rb, amrex::CoordSys::cartesian, per);
}

template <int NC> amrex::Vector<std::string> comp_names() {
    amrex::Vector<std::string> v;
    for (int c = 0; c < NC; ++c) v.push_back("u" + std::to_string(c));
    return v;
}

/// Builds the integrator of `scheme/precision` around an already-built model.
template <class Model>
IntegratorIface* make_for_model(ts_context* ctx, const ts_wave_desc& d, Model&& model, double* table) {
    using M = std::decay_t<Model>;
    constexpr int NC = M::ncomp;
    if (d.scheme == TS_EULER) {
        if (d.precision != TS_PRECISION_F64) throw std::invalid_argument("Euler runs in FP64 only");
        return new Adapter<treesap::SingleLevelEulerIntegrator<M>, NC>(ctx, std::forward<Model>(model), table,
                                                                        kInitTableCap);
    }
    if (d.precision == TS_PRECISION_F32_STAGE) {
        if constexpr (treesap::AffineRHSConcept<typename M::rhs_t>) {
            return new Adapter<treesap::SingleLevelRK4F32StageIntegrator<M>, NC>(ctx, std::forward<Model>(model),
                                                                                  table, kInitTableCap);
        } else {
            throw std::invalid_argument("model is not affine: no FP32-stage form");
        }
    }
    return new Adapter<treesap::SingleLevelRK4Integrator<M>, NC>(ctx, std::forward<Model>(model), table,
                                                                  kInitTableCap);
}

/// PDEModel / ABLPDEModel around an undecorated RHS, optionally KO-decorated (like the oracle).
template <class RHS>
IntegratorIface* make_for_rhs(ts_context* ctx, const ts_wave_desc& d, const RHS& rhs, double* table) {
    constexpr int NC = RHS::ncomp, G = RHS::ngrow;
    using Init = TableInit<NC>;
    const Init init{table};
    const amrex::Geometry geom = geometry_of(d);
    auto with = [&](auto r) -> IntegratorIface* {
        using R = decltype(r);
        if (d.abl_thickness > 0) {
            amrex::GpuArray<amrex::Real, NC> target{};
            for (int c = 0; c < NC; ++c) target[c] = d.bc_values[c];
            auto build = [&](auto profile) -> IntegratorIface* {
                using P = decltype(profile);
                typename treesap::ABLDecorator<R, P>::ABLData abl(target, d.abl_thickness, d.abl_max_strength, profile);
                return make_for_model(ctx, d, treesap::ABLPDEModel<R, Init, P>(comp_names<NC>(), geom, d.dt, r, abl, init),
                                      table);
            };
            if (d.abl_profile == 1) return build(tsb::LinearProfile{});
            return build(tsb::QuadraticProfile{});
        }
        if (d.bc == TS_BC_DIRICHLET) {
            treesap::DirichletBC<NC, G> bc{};
            for (int c = 0; c < NC; ++c) bc.boundary_values[c] = d.bc_values[c];
            return make_for_model(
                ctx, d, treesap::PDEModel<R, Init, treesap::DirichletBC<NC, G>>(comp_names<NC>(), geom, d.dt, r, init, bc),
                table);
        }
        return make_for_model(ctx, d, treesap::PDEModel<R, Init, treesap::NoOpBC<NC, G>>(comp_names<NC>(), geom, d.dt, r, init),
                              table);
    };
    if (d.ko_strength > 0.0) return with(treesap::KODecorator<RHS>{rhs, d.ko_strength});
    return with(rhs);
}

// One per stencil half-width (separate translation units).
// c2 is a device array of c(x)^2 per valid cell (x fastest) or nullptr for unit speed.
IntegratorIface* make_wave_g1(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_wave_g2(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_wave_g3(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_wave_g4(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_wave_adjoint_g2(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_wave_adjoint_g4(ts_context*, const ts_wave_desc&, double* table, const double* c2);
IntegratorIface* make_tensor_f64(ts_context*, const ts_wave_desc&, double* table);
IntegratorIface* make_tensor_f32(ts_context*, const ts_wave_desc&, double* table);

} // namespace treesap_b200
