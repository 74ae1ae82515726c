// Host-only check of the AMReX plotfile writer (util/PlotExporter.hpp): writes a plotfile of a
// known 3-component field into argv[1] (built with g++ against the compat AMReX layer).
#include "util/PlotExporter.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    amrex::Box dom{{0, 0, 0}, {6, 4, 3}};
    amrex::RealBox rb{{-1.0, 0.0, 0.5}, {1.0, 2.0, 1.5}};
    int per[3] = {1, 0, 0};
    amrex::Geometry geom(dom, &rb, amrex::CoordSys::cartesian, per);
    const int n0 = 7, n1 = 5, n2 = 4, nc = 3;
    std::vector<double> v(std::size_t(nc) * n0 * n1 * n2);
    for (int c = 0; c < nc; ++c)
        for (int k = 0; k < n2; ++k)
            for (int j = 0; j < n1; ++j)
                for (int i = 0; i < n0; ++i)
                    v[((std::size_t(c) * n2 + k) * n1 + j) * n0 + i] = 1000.0 * c + 100.0 * k + 10.0 * j + i + 0.25;
    treesap::write_single_level_plotfile(argv[1], v.data(), geom, {"phi", "pi", "speed"}, 0.125, 42);
    return 0;
}
