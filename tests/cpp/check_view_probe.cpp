// Host check of the bounds-checked stencil view (TREESAP_B200_CHECK): an Array4 read through a
// StencilView inside its shared-memory plane and global ranges leaves the error word clear and
// returns the element; a read outside either range sets bit 2 of the error word and returns the
// centre element instead of touching memory outside the buffers. Prints one JSON line.
#define TREESAP_B200_CHECK 1
#include <AMReX.H>

#include <cstdio>

int main() {
    double plane[5 * 7];     // one component, 7 rows of 5, centre at (2, 3)
    double glob[5 * 7 * 9];  // 9 planes of the same shape, centre plane 4
    for (int q = 0; q < 35; ++q) plane[q] = q;
    for (int q = 0; q < 315; ++q) glob[q] = 1000 + q;
    const int pc = 3 * 5 + 2;
    const long long gc = 4 * 35 + pc;
    int err = 0;
    amrex::StencilView<double> v{};
    v.plane = plane + pc;
    v.queue = nullptr;
    v.glob = glob + gc;
    v.gjs = 5;
    v.gks = 35;
    v.gns = 315;
    v.ci = 10;
    v.cj = 20;
    v.ck = 30;
    v.pjs = 5;
    v.pns = 35;
    v.qg = 0;
    v.qnc = 0;
    v.err = &err;
    v.plo = -pc;
    v.phi = 35 - pc;
    v.glo = -gc;
    v.ghi = 315 - gc;
    amrex::Array4<const double> a(glob, amrex::Dim3{0, 0, 0}, amrex::Dim3{5, 7, 9}, 1);
    a.view = &v;
    const double in_plane = a(12, 23, 30, 0);  // (+2, +3) in the plane: index pc + 17 = 34
    const double in_glob = a(11, 21, 34, 0);   // (+1, +1, +4) in global memory
    const int err_in = err;
    const double out_plane = a(13, 23, 30, 0); // (+3, +3): past the plane's end
    const int err_plane = err;
    err = 0;
    const double out_glob = a(10, 20, 35, 0);  // +5 planes: past the field's end
    const int err_glob = err;
    std::printf("{\"in_plane\": %g, \"in_glob\": %g, \"err_in\": %d, \"out_plane\": %g, \"err_plane\": %d, "
                "\"out_glob\": %g, \"err_glob\": %d}\n",
                in_plane, in_glob, err_in, out_plane, err_plane, out_glob, err_glob);
    return 0;
}
