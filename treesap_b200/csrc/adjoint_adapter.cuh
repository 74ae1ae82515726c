// treesap-b200 C ABI: type-erased adapter from ts_adjoint to treesap::WaveAdjointRK4.
#pragma once

#include <treesap_b200.h>

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
};

template <int G> class AdjointAdapter final : public AdjointIface {
  public:
    AdjointAdapter(ts_context* ctx, const ts_wave_desc& d, int every)
        : a_(geometry_of(d), d.dt, d.ko_strength, every, ctx) {}
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

  private:
    treesap::WaveAdjointRK4<G> a_;
};

AdjointIface* make_adjoint_g2(ts_context*, const ts_wave_desc&, int every);
AdjointIface* make_adjoint_g4(ts_context*, const ts_wave_desc&, int every);

} // namespace treesap_b200
