// treesap-b200 C ABI: discrete adjoint (ts_adjoint_*). See include/treesap_b200.h.
#include <cuda_runtime.h>

#include <exception>
#include <stdexcept>
#include <string>

#include "adjoint_adapter.cuh"
#include "runtime_internal.hpp"

struct ts_adjoint {
    ts_context* ctx = nullptr;
    treesap_b200::AdjointIface* impl = nullptr;
};

using namespace treesap_b200;

namespace {

ts_status guarded(ts_context* ctx, const char* what, auto&& fn) {
    try {
        fn();
        return TS_OK;
    } catch (const std::invalid_argument& e) {
        set_error(ctx, std::string(what) + ": " + e.what());
        return TS_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        set_error(ctx, std::string(what) + ": " + e.what());
        const std::string m = e.what();
        return m.find("out of memory") != std::string::npos ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA;
    }
}

} // namespace

extern "C" {

ts_status ts_adjoint_create(ts_context* ctx, const ts_wave_desc* d, int checkpoint_every, ts_adjoint** out) {
    if (!ctx || !out || !d || checkpoint_every < 1) return TS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    for (int q = 0; q < 3; ++q)
        if (d->n[q] < d->ngrow || d->n[q] < 1 || !(d->prob_hi[q] > d->prob_lo[q])) return TS_ERR_INVALID_ARGUMENT;
    if (!(d->dt > 0.0) || d->ko_strength < 0.0) return TS_ERR_INVALID_ARGUMENT;
    if (d->model != TS_MODEL_WAVE || (d->ngrow != 2 && d->ngrow != 4) || d->scheme != TS_RK4 ||
        d->precision != TS_PRECISION_F64 || d->abl_thickness > 0 || !d->periodic[0] || !d->periodic[1] ||
        !d->periodic[2])
        return TS_ERR_UNSUPPORTED;
    auto* a = new ts_adjoint();
    a->ctx = ctx;
    ts_status st = guarded(ctx, "ts_adjoint_create", [&] {
        a->impl = d->ngrow == 2 ? make_adjoint_g2(ctx, *d, checkpoint_every) : make_adjoint_g4(ctx, *d, checkpoint_every);
    });
    if (st != TS_OK) {
        ts_adjoint_destroy(a);
        return st;
    }
    *out = a;
    return TS_OK;
}

ts_status ts_adjoint_destroy(ts_adjoint* a) {
    if (!a) return TS_OK;
    if (a->impl) cudaStreamSynchronize(a->impl->stream());
    delete a->impl;
    delete a;
    return TS_OK;
}

ts_status ts_adjoint_forward(ts_adjoint* a, const double* phi0, const double* pi0, const double* c, int nsteps,
                             double* phi_T, double* pi_T) {
    if (!a || !a->impl || !phi0 || !c || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    return guarded(a->ctx, "ts_adjoint_forward", [&] { a->impl->forward(phi0, pi0, c, nsteps, phi_T, pi_T); });
}

ts_status ts_adjoint_gradient(ts_adjoint* a, const double* phi0, const double* pi0, const double* c, int nsteps,
                              const double* phi_target, double* loss, double* grad_phi0, double* grad_pi0,
                              double* grad_c) {
    if (!a || !a->impl || !phi0 || !c || !phi_target || nsteps < 1) return TS_ERR_INVALID_ARGUMENT;
    return guarded(a->ctx, "ts_adjoint_gradient", [&] {
        const double l = a->impl->gradient(phi0, pi0, c, nsteps, phi_target, grad_phi0, grad_pi0, grad_c);
        if (loss) *loss = l;
    });
}

ts_status ts_adjoint_gradient_f32(ts_adjoint* a, const double* phi0, const double* pi0, const double* c, int nsteps,
                                  const double* phi_target, double* loss, double* grad_phi0, double* grad_pi0,
                                  double* grad_c) {
    if (!a || !a->impl || !phi0 || !c || !phi_target || nsteps < 1) return TS_ERR_INVALID_ARGUMENT;
    return guarded(a->ctx, "ts_adjoint_gradient_f32", [&] {
        const double l = a->impl->gradient_f32(phi0, pi0, c, nsteps, phi_target, grad_phi0, grad_pi0, grad_c);
        if (loss) *loss = l;
    });
}

ts_status ts_adjoint_tangent(ts_adjoint* a, const double* phi0, const double* pi0, const double* c,
                             const double* dphi0, const double* dpi0, const double* dc, int nsteps, double* dphi_T,
                             double* dpi_T) {
    if (!a || !a->impl || !phi0 || !c || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    return guarded(a->ctx, "ts_adjoint_tangent",
                   [&] { a->impl->tangent(phi0, pi0, c, dphi0, dpi0, dc, nsteps, dphi_T, dpi_T); });
}

} // extern "C"
