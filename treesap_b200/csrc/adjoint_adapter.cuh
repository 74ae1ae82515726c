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
    virtual double state_gradient_f32(const double* phi0, const double* pi0, const double* c, int nsteps,
                                      const double* target, double* gphi, double* gpi) = 0;
};

template <int G> class AdjointAdapter final : public AdjointIface {
  public:
    AdjointAdapter(ts_context* ctx, const ts_wave_desc& d, int every)
        : a_(geometry_of(d), d.dt, d.ko_strength, every, ctx), ctx_(ctx), desc_(d) {}
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

    /// FP32-stage form of J and of its gradient with respect to the initial state: the forward
    /// run and the reverse sweep (RK4 with the transposed operator, which does not depend on
    /// the forward states, so no checkpoints are needed) both run in the FP32-stage RK4 form,
    /// on the library's variable-speed wave model and on WaveAdjointSpeedRHS.
    double state_gradient_f32(const double* phi0, const double* pi0, const double* c, int nsteps,
                              const double* target, double* gphi, double* gpi) override {
        const long long ncell = a_.cells();
        struct DevBuf {
            double* p = nullptr;
            ~DevBuf() {
                if (p) cudaFree(p);
            }
        } c2, table;
        std::vector<double> host(std::size_t(ncell) * 2);
        for (long long q = 0; q < ncell; ++q) host[q] = c[q] * c[q];
        cuda_check(cudaMalloc(&c2.p, sizeof(double) * std::size_t(ncell)), "cudaMalloc(c2)");
        cuda_check(cudaMemcpy(c2.p, host.data(), sizeof(double) * std::size_t(ncell), cudaMemcpyHostToDevice),
                   "cudaMemcpy(c2)");
        cuda_check(cudaMalloc(&table.p, sizeof(double) * kInitTableCap), "cudaMalloc(init table)");
        cuda_check(cudaMemset(table.p, 0, sizeof(double) * kInitTableCap), "cudaMemset(init table)"); // no items
        ts_wave_desc d = desc_;
        d.precision = TS_PRECISION_F32_STAGE;
        d.scheme = TS_RK4;
        d.c2 = nullptr;
        std::unique_ptr<IntegratorIface> fwd(G == 2 ? make_wave_g2(ctx_, d, table.p, c2.p)
                                                    : make_wave_g4(ctx_, d, table.p, c2.p));
        for (long long q = 0; q < ncell; ++q) {
            host[q] = phi0[q];
            host[ncell + q] = pi0 ? pi0[q] : 0.0;
        }
        fwd->set_state(host.data(), false);
        for (int st = 0; st < nsteps; ++st) fwd->step();
        fwd->get_state(host.data(), false);
        double loss = 0.0;
        for (long long q = 0; q < ncell; ++q) {
            const double r = host[q] - target[q];
            loss += 0.5 * r * r;
            host[q] = r;
            host[ncell + q] = 0.0;
        }
        std::unique_ptr<IntegratorIface> rev(G == 2 ? make_wave_adjoint_g2(ctx_, d, table.p, c2.p)
                                                    : make_wave_adjoint_g4(ctx_, d, table.p, c2.p));
        rev->set_state(host.data(), false);
        for (int st = 0; st < nsteps; ++st) rev->step();
        rev->get_state(host.data(), false);
        if (gphi) std::copy(host.begin(), host.begin() + ncell, gphi);
        if (gpi) std::copy(host.begin() + ncell, host.end(), gpi);
        return loss;
    }

  private:
    treesap::WaveAdjointRK4<G> a_;
    ts_context* ctx_;
    ts_wave_desc desc_;
};

AdjointIface* make_adjoint_g2(ts_context*, const ts_wave_desc&, int every);
AdjointIface* make_adjoint_g4(ts_context*, const ts_wave_desc&, int every);

} // namespace treesap_b200
