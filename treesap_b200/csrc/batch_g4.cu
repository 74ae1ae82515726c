// treesap-b200 C ABI: batched scalar wave model, stencil half-width 4.
#include "batch_adapter.cuh"

namespace treesap_b200 {

BatchIface* make_batch_g4(ts_context* ctx, const ts_wave_desc* d, int count, double* tables) {
    return make_batch_for_rhs<tsb::WaveRHS<4>>(ctx, d, count, tables);
}

} // namespace treesap_b200
