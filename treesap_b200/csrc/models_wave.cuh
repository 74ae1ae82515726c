// treesap-b200 C ABI: instantiation of the scalar wave models for one stencil half-width
// (TSB_G), included by models_wave_g<N>.cu so the widths compile in parallel.
#include "integrator_adapter.cuh"
#include "WaveAdjointRHS.hpp"

#ifndef TSB_G
#error "define TSB_G before including models_wave.cuh"
#endif

#define TSB_CAT2(a, b) a##b
#define TSB_CAT(a, b) TSB_CAT2(a, b)

namespace treesap_b200 {

IntegratorIface* TSB_CAT(make_wave_g, TSB_G)(ts_context* ctx, const ts_wave_desc& d, double* table, const double* c2) {
    if (c2) {
        tsb::WaveRHS<TSB_G, tsb::FieldSpeed<double>> rhs{};
        rhs.speed = tsb::FieldSpeed<double>{c2, d.n[0], (long long)d.n[0] * d.n[1]};
        return make_for_rhs(ctx, d, rhs, table);
    }
    return make_for_rhs(ctx, d, tsb::WaveRHS<TSB_G>{}, table);
}

#if TSB_G == 2 || TSB_G == 4
/// The transposed wave operator with the speed as a coefficient field (WaveAdjointSpeedRHS,
/// periodic grid, Kreiss-Oliger strength from the descriptor), for the FP32-stage reverse
/// sweep of ts_adjoint_gradient_f32. c2: device array of c(x)^2 per valid cell.
IntegratorIface* TSB_CAT(make_wave_adjoint_g, TSB_G)(ts_context* ctx, const ts_wave_desc& d, double* table,
                                                     const double* c2) {
    tsb::WaveAdjointSpeedRHS<TSB_G> rhs{};
    rhs.c2 = c2;
    for (int q = 0; q < 3; ++q) rhs.n[q] = d.n[q];
    rhs.ko_strength = d.ko_strength;
    using Init = TableInit<2>;
    using M = treesap::PDEModel<tsb::WaveAdjointSpeedRHS<TSB_G>, Init, treesap::NoOpBC<2, TSB_G>>;
    return make_for_model(ctx, d, M(comp_names<2>(), geometry_of(d), d.dt, rhs, Init{table}), table);
}
#endif

} // namespace treesap_b200
