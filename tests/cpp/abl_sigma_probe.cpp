// Host check of the absorbing layer's damping strength: ABLDecorator with QuadraticProfile (which
// offers of_square, so sigma comes from the squared index distance without a square root or a
// branch) against the same profile without of_square (the reference's path: square root, then
// the profile), at every cell of a 64^3 domain with a 16-cell layer. Prints one JSON line: the
// largest relative difference in the layer, and whether both are exactly 0 in the bulk.
#include <AMReX.H>

#include <cmath>
#include <cstdio>

#include "InitFunctors.hpp"
#include "pde-model/rhs-decorators/ABLDecorator.hpp"
#include "pde-model/rhs-decorators/NoOpRHS.hpp"

struct QuadraticOnly {  // s -> s^2 without of_square
    constexpr amrex::Real operator()(amrex::Real s) const { return s * s; }
};

int main() {
    const int n = 64, th = 16;
    amrex::Box dom{{0, 0, 0}, {n - 1, n - 1, n - 1}};
    amrex::RealBox rb{{0.0, 0.0, 0.0}, {1.0, 1.0, 1.0}};
    int per[3] = {0, 0, 0};
    const amrex::Geometry geom(dom, &rb, amrex::CoordSys::cartesian, per);
    using R = treesap::NoOpRHS<1, 1>;
    amrex::GpuArray<amrex::Real, 1> target{0.0};
    const treesap::ABLDecorator<R, tsb::QuadraticProfile> fast(
        R{}, geom, {target, th, 10.0, tsb::QuadraticProfile{}});
    const treesap::ABLDecorator<R, QuadraticOnly> ref(R{}, geom, {target, th, 10.0, QuadraticOnly{}});
    double worst = 0.0;
    long long layer = 0;
    bool bulk_zero = true;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const amrex::IntVect idx{i, j, k};
                const double a = fast.sigma(idx), b = ref.sigma(idx);
                if (b == 0.0) {
                    bulk_zero = bulk_zero && a == 0.0;
                    continue;
                }
                ++layer;
                worst = std::fmax(worst, std::fabs(a - b) / b);
            }
    std::printf("{\"worst_rel\": %.3e, \"layer_cells\": %lld, \"bulk_zero\": %s}\n", worst, layer,
                bulk_zero ? "true" : "false");
    return 0;
}
