// treesap-b200 C ABI: batched scalar wave model, stencil half-width 2.
#include "batch_adapter.cuh"

namespace treesap_b200 {

BatchIface* make_batch_g2(ts_context* ctx, const ts_wave_desc* d, int count, double* tables) {
    return make_batch_for_rhs<tsb::WaveRHS<2>>(ctx, d, count, tables);
}

} // namespace treesap_b200
