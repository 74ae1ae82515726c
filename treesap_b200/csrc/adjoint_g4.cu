// treesap-b200 C ABI: discrete adjoint of the variable-speed wave model, stencil half-width 4.
#include "adjoint_adapter.cuh"

namespace treesap_b200 {

AdjointIface* make_adjoint_g4(ts_context* ctx, const ts_wave_desc& d, int every) {
    return new AdjointAdapter<4>(ctx, d, every);
}

} // namespace treesap_b200
