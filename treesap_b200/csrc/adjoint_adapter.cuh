// treesap-b200 C ABI: type-erased adapter from ts_adjoint to treesap::WaveAdjointRK4.
#pragma once

#include <treesap_b200.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "integrator_adapter.cuh"
#include "integrators/WaveAdjointRK4.hpp"

namespace treesap_b200 {

struct AdjointIface {
    virtual ~AdjointIface() = default;
    virtual long long cells() const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual void forward(const double* phi0, const double* pi0, const double* c, int nsteps, double* phiT,
                         double* piT) = 0;
    virtual double gradient(const double* phi0, const double* pi0, const double* c, int nsteps, const double* target,
                            double* gphi, double* gpi, double* gc) = 0;
    virtual void tangent(const double* phi0, const double* pi0, const double* c, const double* dphi0,
                         const double* dpi0, const double* dc, int nsteps, double* dphiT, double* dpiT) = 0;
    virtual double gradient_f32(const double* phi0, const double* pi0, const double* c, int nsteps,
                                const double* target, double* gphi, double* gpi, double* gc) = 0;
};

template <int G> class AdjointAdapter final : public AdjointIface {
  public:
    AdjointAdapter(ts_context* ctx, const ts_wave_desc& d, int every)
        : a_(geometry_of(d), d.dt, d.ko_strength, every, ctx), ctx_(ctx), desc_(d), every_(every) {}
    long long cells() const override { return a_.cells(); }
    cudaStream_t stream() const override { return a_.stream(); }
    void forward(const double* phi0, const double* pi0, const double* c, int nsteps, double* phiT,
                 double* piT) override {
        a_.forward(phi0, pi0, c, nsteps, phiT, piT);
    }
    double gradient(const double* phi0, const double* pi0, const double* c, int nsteps, const double* target,
                    double* gphi, double* gpi, double* gc) override {
        return a_.gradient(phi0, pi0, c, nsteps, target, gphi, gpi, gc);
    }
    void tangent(const double* phi0, const double* pi0, const double* c, const double* dphi0, const double* dpi0,
                 const double* dc, int nsteps, double* dphiT, double* dpiT) override {
        a_.tangent(phi0, pi0, c, dphi0, dpi0, dc, nsteps, dphiT, dpiT);
    }

    /// FP32-stage form of J and of its gradients. The forward run and the reverse sweep (RK4
    /// with the transposed operator) both run in the FP32-stage RK4 form, on the library's
    /// variable-speed wave model and on WaveAdjointSpeedRHS. The state gradient needs only the
    /// reverse sweep (the transposed operator does not depend on the forward states). The speed
    /// gradient (gc non-null) needs each forward step's registers: the forward states are kept
    /// every `checkpoint_every` steps, each segment is recomputed from its checkpoint, and per
    /// step of the reverse sweep the forward step (u, k0, d1, d2) and the adjoint step run
    /// stage by stage before the four gradient terms (WaveSpeedGradientF32) are added.
    /// The two integrators and the device buffers are built on the first call and reused.
    double gradient_f32(const double* phi0, const double* pi0, const double* c, int nsteps, const double* target,
                        double* gphi, double* gpi, double* gc) override {
        const long long ncell = a_.cells();
        F32State& f = f32_state();
        cudaStream_t s = a_.stream();
        std::vector<double>& host = f.host;
        for (long long q = 0; q < ncell; ++q) host[q] = c[q] * c[q];
        // c^2 is read by both models through their device pointer
        cuda_check(cudaMemcpyAsync(f.c2.p, host.data(), sizeof(double) * std::size_t(ncell), cudaMemcpyHostToDevice, s),
                   "cudaMemcpyAsync(c2)");
        cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize(c2)");
        IntegratorIface* fwd = f.fwd.get();
        IntegratorIface* rev = f.rev.get();
        StageOps* fops = fwd->stage_ops();
        StageOps* rops = rev->stage_ops();
        if (gc && (!fops || !rops)) throw std::logic_error("FP32-stage integrators without stage-level stepping");
        const long long sz = 2 * ncell; // one packed two-component state
        const int nck = gc ? (nsteps + every_ - 1) / every_ : 0;
        if (gc) {
            const std::size_t states = std::size_t(nck) + std::size_t(every_);
            if (states > f.store_states) {
                f.store = DevBuf{};
                cuda_check(cudaMalloc(&f.store.p, sizeof(double) * std::size_t(sz) * states), "cudaMalloc(checkpoints)");
                f.store_states = states;
            }
        }
        double* store = f.store.p;
        auto ckpt = [&](int i) { return store + std::size_t(i) * sz; };
        auto seg = [&](int m) { return store + std::size_t(nck + m) * sz; };
        for (long long q = 0; q < ncell; ++q) {
            host[q] = phi0[q];
            host[ncell + q] = pi0 ? pi0[q] : 0.0;
        }
        fwd->set_state(host.data(), false);
        for (int st = 0; st < nsteps; ++st) {
            if (gc && st % every_ == 0) fwd->get_state(ckpt(st / every_), true);
            fwd->step();
        }
        fwd->get_state(host.data(), false);
        double loss = 0.0;
        for (long long q = 0; q < ncell; ++q) {
            const double r = host[q] - target[q];
            loss += 0.5 * r * r;
            host[q] = r;
            host[ncell + q] = 0.0;
        }
        rev->set_state(host.data(), false);
        if (!gc) {
            for (int st = 0; st < nsteps; ++st) rev->step();
        } else {
            DeviceField<double>& g = *f.g;
            cuda_check(cudaMemsetAsync(g.data(), 0, std::size_t(g.layout().bytes()), s), "cudaMemsetAsync(gradient)");
            using Reg = typename treesap::WaveSpeedGradientF32<G>::Reg;
            for (int sg = nck - 1; sg >= 0; --sg) {
                const int start = sg * every_, end = std::min(nsteps, start + every_);
                fwd->set_state(ckpt(sg), true);
                for (int m = 1; m < end - start; ++m) {
                    fwd->step();
                    fwd->get_state(seg(m), true);
                }
                for (int st = end - 1; st >= start; --st) {
                    const int m = st - start;
                    fwd->set_state(m == 0 ? ckpt(sg) : seg(m), true);
                    Reg fr[4], ar[4];
                    for (int q = 0; q < 4; ++q) fops->run_stage(q);
                    for (int q = 0; q < 4; ++q) rops->run_stage(q);
                    for (int q = 0; q < 4; ++q) {
                        fops->field(q, &fr[q].data, &fr[q].L);
                        rops->field(q, &ar[q].data, &ar[q].L);
                    }
                    f.grad->accumulate(fr, ar, g.data(), g.layout(), desc_.dt);
                    rops->finish();
                    fops->finish();
                }
            }
            // the valid cells of g into the first checkpoint slot, then to the host
            launch_pack(g.data(), g.layout(), store, 1, ts_context_sm_count(ctx_), s);
            cuda_check(cudaMemcpyAsync(gc, store, sizeof(double) * std::size_t(ncell), cudaMemcpyDeviceToHost, s),
                       "cudaMemcpyAsync(speed gradient)");
            cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize(speed gradient)");
            for (long long q = 0; q < ncell; ++q) gc[q] *= 2.0 * c[q];
        }
        rev->get_state(host.data(), false);
        if (gphi) std::copy(host.begin(), host.begin() + ncell, gphi);
        if (gpi) std::copy(host.begin() + ncell, host.end(), gpi);
        return loss;
    }

  private:
    struct DevBuf {
        double* p = nullptr;
        DevBuf() = default;
        DevBuf(const DevBuf&) = delete;
        DevBuf& operator=(const DevBuf&) = delete;
        DevBuf& operator=(DevBuf&& o) noexcept {
            if (this != &o) {
                if (p) cudaFree(p);
                p = o.p;
                o.p = nullptr;
            }
            return *this;
        }
        ~DevBuf() {
            if (p) cudaFree(p);
        }
    };
    /// The FP32-stage form's integrators and buffers (built by the first gradient_f32 call).
    struct F32State {
        DevBuf c2, table, store;
        std::size_t store_states = 0;
        std::vector<double> host;
        std::unique_ptr<IntegratorIface> fwd, rev;
        std::unique_ptr<DeviceField<double>> g;
        std::unique_ptr<treesap::WaveSpeedGradientF32<G>> grad;
    };
    F32State& f32_state() {
        if (f32_) return *f32_;
        auto f = std::make_unique<F32State>();
        const long long ncell = a_.cells();
        f->host.resize(std::size_t(ncell) * 2);
        cuda_check(cudaMalloc(&f->c2.p, sizeof(double) * std::size_t(ncell)), "cudaMalloc(c2)");
        cuda_check(cudaMalloc(&f->table.p, sizeof(double) * kInitTableCap), "cudaMalloc(init table)");
        cuda_check(cudaMemset(f->table.p, 0, sizeof(double) * kInitTableCap), "cudaMemset(init table)"); // no items
        ts_wave_desc d = desc_;
        d.precision = TS_PRECISION_F32_STAGE;
        d.scheme = TS_RK4;
        d.c2 = nullptr;
        f->fwd.reset(G == 2 ? make_wave_g2(ctx_, d, f->table.p, f->c2.p) : make_wave_g4(ctx_, d, f->table.p, f->c2.p));
        f->rev.reset(G == 2 ? make_wave_adjoint_g2(ctx_, d, f->table.p, f->c2.p)
                            : make_wave_adjoint_g4(ctx_, d, f->table.p, f->c2.p));
        const int n[3] = {desc_.n[0], desc_.n[1], desc_.n[2]};
        f->g = std::make_unique<DeviceField<double>>(n, G, 1);
        f->grad = std::make_unique<treesap::WaveSpeedGradientF32<G>>(ctx_, geometry_of(d).data());
        f32_ = std::move(f);
        return *f32_;
    }

    treesap::WaveAdjointRK4<G> a_;
    ts_context* ctx_;
    ts_wave_desc desc_;
    int every_;
    std::unique_ptr<F32State> f32_; // destroyed before a_ (declared after it)
};

AdjointIface* make_adjoint_g2(ts_context*, const ts_wave_desc&, int every);
AdjointIface* make_adjoint_g4(ts_context*, const ts_wave_desc&, int every);

} // namespace treesap_b200
