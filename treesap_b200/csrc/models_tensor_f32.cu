// treesap-b200 C ABI: the tensorial wave model (12 components, TensorWaveRHS.hpp) in the
// configuration it is benchmarked in: stencil half-width 3, Kreiss-Oliger, no absorbing layer,
// NoOp boundary functor (periodic directions take periodic images), RK4 (f32 form).
// The 12-component kernels compile for minutes each, so only this configuration is built.
#include "integrator_adapter.cuh"

namespace treesap_b200 {

IntegratorIface* make_tensor_f32(ts_context* ctx, const ts_wave_desc& d, double* table) {
    using R = treesap::KODecorator<tsb::TensorWaveRHS<3>>;
    using Init = TableInit<12>;
    using M = treesap::PDEModel<R, Init, treesap::NoOpBC<12, 3>>;
    M model(comp_names<12>(), geometry_of(d), d.dt, R{tsb::TensorWaveRHS<3>{}, d.ko_strength}, Init{table});
    return new Adapter<treesap::SingleLevelRK4F32StageIntegrator<M>, 12>(ctx, std::move(model), table, kInitTableCap);
}

} // namespace treesap_b200
