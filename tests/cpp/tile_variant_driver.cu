// Runs the 8th-order wave model with Kreiss-Oliger dissipation and an absorbing layer
// (Dirichlet ghosts) on a ragged box through the front end, FP64 RK4 and the FP32-stage form,
// and writes both final states (FP64 valid cells, [form][comp][z][y][x]) to argv[1]. Built
// once per stage-kernel tile configuration (-DTREESAP_B200_TILE_F64=..., -DTREESAP_B200_QROT_F64=...):
// the per-cell arithmetic does not depend on the tiling, so every build must write the same bytes.
#include <AMReX.H>

#include <cstdio>
#include <vector>

#include "integrators/SingleLevelRK4F32StageIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "pde-model/ABLPDEModel.hpp"
#include "pde-model/rhs-decorators/KODecorator.hpp"

#include "InitFunctors.hpp"
#include "WaveRHS.hpp"

using RHS = treesap::KODecorator<tsb::WaveRHS<4>>;
using Init = tsb::GaussianSumInit<2>;
using Model = treesap::ABLPDEModel<RHS, Init, tsb::QuadraticProfile>;

static const int kN[3] = {72, 45, 37};

static Model make_model() {
    amrex::Box dom{{0, 0, 0}, {kN[0] - 1, kN[1] - 1, kN[2] - 1}};
    amrex::RealBox rb{{0.0, 0.0, 0.0}, {1.0, 45.0 / 72.0, 37.0 / 72.0}};
    int per[3] = {0, 0, 0};
    amrex::Geometry geom(dom, &rb, amrex::CoordSys::cartesian, per);
    Init init{};
    init.npulses = 3;
    const double p[3][5] = {{1.0, 0.08, 0.4, 0.3, 0.25}, {0.7, 0.05, 0.6, 0.35, 0.2}, {0.5, 0.1, 0.5, 0.2, 0.3}};
    for (int q = 0; q < 3; ++q) {
        init.comp[q] = 0;
        init.amp[q] = p[q][0];
        init.width[q] = p[q][1];
        init.cx[q] = p[q][2];
        init.cy[q] = p[q][3];
        init.cz[q] = p[q][4];
    }
    amrex::GpuArray<amrex::Real, 2> target{0.0, 0.0};
    treesap::ABLDecorator<RHS, tsb::QuadraticProfile>::ABLData abl(target, 6, 10.0, tsb::QuadraticProfile{});
    return Model({"phi", "pi"}, geom, 0.25 / kN[0], RHS{tsb::WaveRHS<4>{}, 0.2}, abl, init);
}

template <class Integ> void run(std::vector<double>& out, int steps) {
    Integ it(make_model(), amrex::IntVect{1 << 30, 1 << 30, 1 << 30});
    it.initialise();
    for (int s = 0; s < steps; ++s) it.step();
    const std::size_t n = std::size_t(kN[0]) * kN[1] * kN[2] * 2;
    std::vector<double> h(n);
    it.get_state(h.data());
    out.insert(out.end(), h.begin(), h.end());
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    amrex::Initialize(argc, argv);
    std::vector<double> all;
    {
        run<treesap::SingleLevelRK4Integrator<Model>>(all, 12);
        run<treesap::SingleLevelRK4F32StageIntegrator<Model>>(all, 12);
    }
    // the device error word must be clear (checked builds record out-of-range indices there)
    const ts_status st = ts_context_sync(treesap_b200::default_context());
    amrex::Finalize();
    if (st != TS_OK) {
        std::fprintf(stderr, "device error: %s\n", ts_context_last_error(treesap_b200::default_context()));
        return 5;
    }
    FILE* f = std::fopen(argv[1], "wb");
    if (!f) return 3;
    const bool ok = std::fwrite(all.data(), sizeof(double), all.size(), f) == all.size();
    std::fclose(f);
    return ok ? 0 : 4;
}
