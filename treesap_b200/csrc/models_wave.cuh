// treesap-b200 C ABI: instantiation of the scalar wave models for one stencil half-width
// (TSB_G), included by models_wave_g<N>.cu so the widths compile in parallel.
#include "integrator_adapter.cuh"

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

} // namespace treesap_b200
