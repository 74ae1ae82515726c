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

#include "integrators/SingleLevelDOPRI5Integrator.hpp"
#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4F32StageIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "integrators/ZSlabDomain.hpp"
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

/// Stage-level operations of one z slab of a domain shared by several processes (ts_slab_*).
struct SlabOps {
    virtual ~SlabOps() = default;
    virtual int stages() const = 0;
    virtual void prepare(int s) = 0;
    /// The ngrow boundary planes sent to the neighbour across `face` (0 lower, 1 upper): whole
    /// planes from component 0, `elems` elements of `esize` bytes per component, components `cs`
    /// elements apart.
    virtual void send_planes(int s, int face, void** ptr, long long* elems, long long* cs, int* esize) = 0;
    /// Copies received planes (ncomp blocks of `elems` elements) into the ghost planes of `face`.
    virtual void receive_planes(int s, int face, const void* buf) = 0;
    virtual void fill(int s) = 0;
    virtual void launch(int s) = 0;
    virtual void finish() = 0;
};

/// A slab request for the next model built on this host thread (ts_integrator_create_slab):
/// make_for_model then builds the slab's integrator instead of a whole-domain one.
struct SlabRequest {
    bool active = false;
    SlabZ sz{};
    int depth = 0;
};
inline SlabRequest& slab_request() {
    static thread_local SlabRequest r;
    return r;
}

/// Stage-level stepping of a whole-domain RK4-family integrator with access to its stage
/// registers: after run_stage(s), field(s) is the input of stage s with its ghost cells filled
/// (FP32-stage form: u, k0, d1, d2), valid until finish() ends the step.
struct StageOps {
    virtual ~StageOps() = default;
    virtual int stages() const = 0;
    virtual void run_stage(int s) = 0;
    virtual void finish() = 0;
    virtual void field(int s, void** data, Layout* L) = 0;
};

struct IntegratorIface {
    virtual ~IntegratorIface() = default;
    virtual SlabOps* slab_ops() { return nullptr; }
    virtual StageOps* stage_ops() { return nullptr; }
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
    virtual void adaptive_stats(long long*, long long*, double*, double*) {
        throw std::invalid_argument("not an adaptive (TS_DOPRI5) integrator");
    }
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

template <class Integ, int NC> class Adapter final : public IntegratorIface, public StageOps {
    static constexpr bool kStageApi = requires(Integ& i) { i.stage_launch(0, 0.0); };

  public:
    template <class Model, class... Extra>
    Adapter(ts_context* ctx, Model&& model, double* table, std::size_t table_cap, Extra... extra)
        : integ_(std::forward<Model>(model), amrex::IntVect{1 << 30, 1 << 30, 1 << 30}, ctx, extra...), table_(table),
          table_cap_(table_cap) {}
    StageOps* stage_ops() override {
        if constexpr (kStageApi) return this;
        return nullptr;
    }
    int stages() const override {
        if constexpr (kStageApi) return Integ::kStages;
        return 0;
    }
    void run_stage(int s) override {
        if constexpr (kStageApi) {
            const double dt = integ_.get_model().dt_hint();
            integ_.stage_prepare(s);
            integ_.stage_fill(s, dt);
            integ_.stage_launch(s, dt);
        }
    }
    void finish() override {
        if constexpr (kStageApi) integ_.stage_finish(integ_.get_model().dt_hint());
    }
    void field(int s, void** data, Layout* L) override {
        if constexpr (kStageApi) {
            const auto f = integ_.stage_ref(s);
            *data = f.data;
            *L = f.L;
        }
    }
    void adaptive_stats(long long* acc, long long* rej, double* next_dt, double* err) override {
        if constexpr (requires { integ_.accepted(); }) {
            *acc = integ_.accepted();
            *rej = integ_.rejected();
            *next_dt = integ_.proposed_dt();
            *err = integ_.last_error();
        } else {
            IntegratorIface::adaptive_stats(acc, rej, next_dt, err);
        }
    }
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

/// A domain split into z slabs (ts_wave_desc.block[2], ZSlabDomain.hpp) behind the same
/// interface; the slabs' initial-condition table is the ts_integrator's.
template <class Integ, int NC> class SlabAdapter final : public IntegratorIface {
  public:
    template <class Model>
    SlabAdapter(ts_context* ctx, Model&& model, int block_z, double* table, std::size_t table_cap)
        : dom_(std::forward<Model>(model), amrex::IntVect{1 << 30, 1 << 30, block_z}, ctx), ctx_(ctx), table_(table),
          table_cap_(table_cap) {}
    int ncomp() const override { return NC; }
    void initialise(int kind, int nitems, const double* items) override {
        if (nitems < 0 || std::size_t(2 + 6 * nitems) > table_cap_) throw std::invalid_argument("too many init items");
        std::vector<double> host(2 + 6 * std::size_t(nitems));
        host[0] = kind;
        host[1] = nitems;
        for (int q = 0; q < 6 * nitems; ++q) host[2 + q] = items[q];
        upload(host);
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
        upload(host);
    }
    void set_state(const double* src, bool dev) override { dom_.set_state(src, dev); }
    void get_state(double* dst, bool dev) override { dom_.get_state(dst, dev); }
    void step() override { dom_.step(); }
    void step_host_only() override { throw std::invalid_argument("CUDA graphs are not built for z-slab domains"); }
    double time() const override { return dom_.time(); }
    long long steps() const override { return dom_.steps(); }
    void* state_ptr() override { return dom_.slab(0).state().data(); }
    Layout state_layout() const override { return const_cast<SlabAdapter*>(this)->dom_.slab(0).state().layout(); }
    long long launches_per_step() const override { return dom_.launches_per_step(); }
    void attach_clock(treesap::KernelClock* c) override { dom_.attach_clock(c); }
    void set_launch_shape(int rows, int chunks) override { dom_.set_launch_shape(rows, chunks); }
    bool state_is_finite() override { return dom_.state_is_finite(); }

  private:
    void upload(const std::vector<double>& host) {
        if (host.size() > table_cap_) throw std::invalid_argument("initial condition too long for the parameter table");
        cudaStream_t s = static_cast<cudaStream_t>(ts_context_stream(ctx_));
        cuda_check(cudaMemcpyAsync(table_, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, s),
                   "cudaMemcpyAsync(init table)");
        dom_.initialise();
        cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize(initialise)");
    }
    treesap::ZSlabDomain<Integ> dom_;
    ts_context* ctx_;
    double* table_;
    std::size_t table_cap_;
};

/// One z slab of a domain decomposed over processes: the whole-domain Adapter interface on the
/// slab's own cells (set/get_state take [comp][z_slab][y][x]) plus its stage-level operations.
template <class Integ, int NC> class RankSlabAdapter final : public IntegratorIface, public SlabOps {
  public:
    template <class Model>
    RankSlabAdapter(ts_context* ctx, Model&& model, const SlabZ& sz, int depth, double* table, std::size_t cap)
        : inner_(ctx, std::forward<Model>(model), table, cap, sz, depth) {}
    SlabOps* slab_ops() override { return this; }
    int ncomp() const override { return NC; }
    void initialise(int kind, int nitems, const double* items) override { inner_.initialise(kind, nitems, items); }
    void initialise_expressions(int count, const char* const* exprs) override {
        inner_.initialise_expressions(count, exprs);
    }
    void set_state(const double* src, bool dev) override { inner_.set_state(src, dev); }
    void get_state(double* dst, bool dev) override { inner_.get_state(dst, dev); }
    void step() override { throw std::invalid_argument("a slab of a shared domain steps through ts_slab_* calls"); }
    void step_host_only() override { step(); }
    double time() const override { return inner_.time(); }
    long long steps() const override { return inner_.steps(); }
    void* state_ptr() override { return inner_.state_ptr(); }
    Layout state_layout() const override { return inner_.state_layout(); }
    long long launches_per_step() const override { return inner_.launches_per_step(); }
    void attach_clock(treesap::KernelClock* c) override { inner_.attach_clock(c); }
    void set_launch_shape(int rows, int chunks) override { inner_.set_launch_shape(rows, chunks); }
    bool state_is_finite() override { return inner_.state_is_finite(); }

    int stages() const override { return Integ::kStages; }
    void prepare(int s) override { integ().stage_prepare(s); }
    void send_planes(int s, int face, void** ptr, long long* elems, long long* cs, int* esize) override {
        const auto f = integ().stage_ref(s);
        const Layout& L = f.L;
        const long long plane = L.px * L.py;
        const int first = face == 0 ? 0 : L.n[2] - L.g; // its lowest / highest ngrow valid planes
        *ptr = static_cast<char*>(f.data) + (long long)(first + L.g) * plane * L.esize;
        *elems = (long long)L.g * plane;
        *cs = L.comp_stride();
        *esize = L.esize;
    }
    void receive_planes(int s, int face, const void* buf) override {
        const auto f = integ().stage_ref(s);
        const Layout& L = f.L;
        const int kd0 = face == 0 ? -L.g : L.n[2];
        const long long cs = (long long)L.g * L.px * L.py;
        if (L.esize == 8)
            launch_halo_copy(static_cast<double*>(f.data), L, kd0, static_cast<const double*>(buf), cs, L.g,
                             integ().sm_count(), integ().stream());
        else
            launch_halo_copy(static_cast<float*>(f.data), L, kd0, static_cast<const float*>(buf), cs, L.g,
                             integ().sm_count(), integ().stream());
    }
    void fill(int s) override { integ().stage_fill(s, integ().get_model().dt_hint()); }
    void launch(int s) override { integ().stage_launch(s, integ().get_model().dt_hint()); }
    void finish() override { integ().stage_finish(integ().get_model().dt_hint()); }

  private:
    /// The whole-domain adapter's services (table upload, state copies) around the slab integrator.
    struct Inner {
        template <class Model>
        Inner(ts_context* ctx, Model&& model, double* table, std::size_t cap, const SlabZ& sz, int depth)
            : integ(std::forward<Model>(model), amrex::IntVect{1 << 30, 1 << 30, 1 << 30}, ctx, sz, depth),
              ctx(ctx), table(table), cap(cap) {}
        Integ integ;
        ts_context* ctx;
        double* table;
        std::size_t cap;
        void upload(const std::vector<double>& host) {
            if (host.size() > cap) throw std::invalid_argument("initial condition too long for the parameter table");
            cuda_check(cudaMemcpyAsync(table, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice,
                                       integ.stream()),
                       "cudaMemcpyAsync(init table)");
            integ.initialise();
            cuda_check(cudaStreamSynchronize(integ.stream()), "cudaStreamSynchronize(initialise)");
        }
        void initialise(int kind, int nitems, const double* items) {
            if (nitems < 0 || std::size_t(2 + 6 * nitems) > cap) throw std::invalid_argument("too many init items");
            std::vector<double> host(2 + 6 * std::size_t(nitems));
            host[0] = kind;
            host[1] = nitems;
            for (int q = 0; q < 6 * nitems; ++q) host[2 + q] = items[q];
            upload(host);
        }
        void initialise_expressions(int count, const char* const* exprs) {
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
            upload(host);
        }
        void set_state(const double* src, bool dev) { integ.set_state(src, dev); }
        void get_state(double* dst, bool dev) { integ.get_state(dst, dev); }
        double time() const { return integ.get_time(); }
        long long steps() const { return (long long)integ.get_steps(); }
        void* state_ptr() { return integ.state().data(); }
        Layout state_layout() const { return integ.state().layout(); }
        long long launches_per_step() const { return integ.launches_per_step(); }
        void attach_clock(treesap::KernelClock* c) { integ.attach_clock(c); }
        void set_launch_shape(int rows, int chunks) { integ.set_launch_shape(rows, chunks); }
        bool state_is_finite() { return integ.state_is_finite(); }
    };
    Integ& integ() { return inner_.integ; }
    Inner inner_;
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
    if (slab_request().active) {
        const SlabRequest r = slab_request();
        if (d.precision == TS_PRECISION_F32_STAGE) {
            if constexpr (treesap::AffineRHSConcept<typename M::rhs_t>) {
                return new RankSlabAdapter<treesap::SingleLevelRK4F32StageIntegrator<M>, NC>(
                    ctx, std::forward<Model>(model), r.sz, r.depth, table, kInitTableCap);
            } else {
                throw std::invalid_argument("model is not affine: no FP32-stage form");
            }
        }
        if (d.scheme == TS_EULER)
            return new RankSlabAdapter<treesap::SingleLevelEulerIntegrator<M>, NC>(ctx, std::forward<Model>(model),
                                                                                r.sz, r.depth, table, kInitTableCap);
        return new RankSlabAdapter<treesap::SingleLevelRK4Integrator<M>, NC>(ctx, std::forward<Model>(model), r.sz,
                                                                           r.depth, table, kInitTableCap);
    }
    if (d.scheme == TS_DOPRI5) {
        if (d.precision != TS_PRECISION_F64 || (d.block[2] > 0 && d.block[2] < d.n[2]))
            throw std::invalid_argument("DOPRI5 runs in FP64 on one box");
        return new Adapter<treesap::SingleLevelDOPRI5Integrator<M>, NC>(ctx, std::forward<Model>(model), table,
                                                                         kInitTableCap, d.rtol > 0.0 ? d.rtol : 1e-6,
                                                                         d.atol > 0.0 ? d.atol : 1e-9);
    }
    if (d.block[2] > 0 && d.block[2] < d.n[2]) {
        if (d.precision == TS_PRECISION_F32_STAGE) {
            if constexpr (treesap::AffineRHSConcept<typename M::rhs_t>) {
                return new SlabAdapter<treesap::SingleLevelRK4F32StageIntegrator<M>, NC>(
                    ctx, std::forward<Model>(model), d.block[2], table, kInitTableCap);
            } else {
                throw std::invalid_argument("model is not affine: no FP32-stage form");
            }
        }
        if (d.scheme == TS_EULER)
            return new SlabAdapter<treesap::SingleLevelEulerIntegrator<M>, NC>(ctx, std::forward<Model>(model),
                                                                            d.block[2], table, kInitTableCap);
        return new SlabAdapter<treesap::SingleLevelRK4Integrator<M>, NC>(ctx, std::forward<Model>(model), d.block[2],
                                                                       table, kInitTableCap);
    }
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
