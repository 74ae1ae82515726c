// A user program of the header front end, written like the reference's example drivers: a
// PDEModel with FunctionInit and Dirichlet boundaries, SingleLevelRK4Integrator, exports every
// 2 steps through configureExporter. argv[1] = export path prefix.
#include <AMReX.H>

#include "init/FunctionInit.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "pde-model/PDEModel.hpp"
#include "pde-model/bcs/DirichletBC.hpp"
#include "util/ScopedTimer.hpp"

#include "WaveRHS.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    amrex::Initialize(argc, argv);
    {
        amrex::Box index_range{{0, 0, 0}, {23, 19, 15}};
        amrex::RealBox coord_range{{0.0, 0.0, 0.0}, {1.0, 1.0, 1.0}};
        int is_per[] = {0, 0, 0};
        amrex::Geometry geom(index_range, &coord_range, amrex::CoordSys::cartesian, is_per);
        const amrex::Real dt = 0.25 / 24;
        using RHSType = tsb::WaveRHS<2>;
        using InitType = treesap::FunctionInit<RHSType::ncomp>;
        using BCType = treesap::DirichletBC<RHSType::ncomp, RHSType::ngrow>;
        using ModelType = treesap::PDEModel<RHSType, InitType, BCType>;
        InitType init({"exp(-((x-0.5)^2 + (y-0.5)^2 + (z-0.5)^2)/0.15^2)", "0.0"});
        BCType bc{0.0, 0.0};
        ModelType model({"phi", "pi"}, std::move(geom), dt, RHSType{}, std::move(init), std::move(bc));
        treesap::SingleLevelRK4Integrator<ModelType> integrator(std::move(model), {8, 8, 8});
        integrator.initialise();
        integrator.configureExporter(argv[1], 2);
        treesap::ScopedTimer::enabled = true;
        for (int step = 0; step <= 4; ++step) integrator.step();
        if (treesap::ScopedTimer::enabled) treesap::ScopedTimer::printOverview();
    }
    amrex::Finalize();
    return 0;
}
