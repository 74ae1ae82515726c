// treesap-b200: periodic export of the state (API of the reference util/PlotExporter.hpp:29-67:
// exportIfNecessary(step, time) writes at step % interval == 0 to path + step zero-padded to 5).
//
// The reference calls amrex::WriteSingleLevelPlotfile. This build has no AMReX, so the writer
// below produces the same on-disk format itself: an AMReX plotfile (text `Header` of version
// HyperCLaw-V1.1, one level, one box covering the domain; `Level_0/Cell_H`, the VisMF header
// with the per-component minima and maxima; `Level_0/Cell_D_00000`, one FAB: a text line
// giving the real format (IEEE double, little-endian), the box and the component count, then
// the valid cells of every component, x fastest). Readers of AMReX plotfiles (yt, Amrvis,
// VisIt) open it like the reference's output. The state is copied from the device once the
// stream reaches the export point.
#pragma once

#include <AMReX.H>

#include <algorithm>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "ScopedTimer.hpp"

namespace treesap {

namespace fs = std::filesystem;

/// Writes one single-level, single-box AMReX plotfile into directory `dir` from the valid cells
/// `data` ([comp][z][y][x], ncomp x n0 n1 n2 doubles).
inline void write_single_level_plotfile(const fs::path& dir, const double* data, const amrex::Geometry& geom,
                                        const amrex::Vector<std::string>& names, amrex::Real time, int step) {
    const amrex::Box& dom = geom.Domain();
    const int n[3] = {dom.length(0), dom.length(1), dom.length(2)};
    const long long ncell = (long long)n[0] * n[1] * n[2];
    const int ncomp = int(names.size());
    fs::create_directories(dir / "Level_0");
    auto box_text = [&] {
        std::ostringstream b;
        b << "((" << dom.smallEnd(0) << "," << dom.smallEnd(1) << "," << dom.smallEnd(2) << ") (" << dom.bigEnd(0)
          << "," << dom.bigEnd(1) << "," << dom.bigEnd(2) << ") (0,0,0))";
        return b.str();
    };
    {
        std::ofstream h(dir / "Header");
        h << std::setprecision(std::numeric_limits<double>::max_digits10);
        h << "HyperCLaw-V1.1\n" << ncomp << "\n";
        for (const auto& s : names) h << s << "\n";
        h << 3 << "\n" << time << "\n" << 0 << "\n"; // space dimension, time, finest level
        for (int d = 0; d < 3; ++d) h << geom.ProbLo(d) << (d < 2 ? " " : "\n");
        for (int d = 0; d < 3; ++d) h << geom.ProbHi(d) << (d < 2 ? " " : "\n");
        h << "\n";                                         // refinement ratios: none for one level
        h << box_text() << "\n" << step << "\n";           // level domain, level step
        for (int d = 0; d < 3; ++d) h << geom.CellSize(d) << (d < 2 ? " " : "\n");
        h << 0 << "\n" << 0 << "\n";                       // coordinate system, boundary width
        h << 0 << " " << 1 << " " << time << "\n" << step << "\n"; // level 0: one grid
        for (int d = 0; d < 3; ++d) h << geom.ProbLo(d) << " " << geom.ProbHi(d) << "\n";
        h << "Level_0/Cell\n";
    }
    {
        std::ofstream d(dir / "Level_0" / "Cell_D_00000", std::ios::binary);
        d << "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))" << box_text() << " " << ncomp << "\n";
        d.write(reinterpret_cast<const char*>(data), std::streamsize(sizeof(double) * ncell * ncomp));
    }
    {
        std::ofstream c(dir / "Level_0" / "Cell_H");
        c << std::setprecision(std::numeric_limits<double>::max_digits10);
        c << 1 << "\n" << 1 << "\n" << ncomp << "\n" << 0 << "\n"; // version, layout, components, ghost width
        c << "(1 0\n" << box_text() << "\n)\n";
        c << 1 << "\n" << "FabOnDisk: Cell_D_00000 0\n\n";
        for (int which = 0; which < 2; ++which) {
            c << 1 << "," << ncomp << "\n";
            for (int q = 0; q < ncomp; ++q) {
                const double* p = data + q * ncell;
                const double v = which == 0 ? *std::min_element(p, p + ncell) : *std::max_element(p, p + ncell);
                c << v << ",";
            }
            c << "\n\n";
        }
    }
}

class PlotExporter {
  public:
    /// `fetch` copies the current valid state (ncomp x ncell doubles) into the given host buffer.
    PlotExporter(std::function<void(double*)> fetch, const amrex::Geometry& geom,
                 const amrex::Vector<std::string>& comp_names, fs::path path, int export_interval)
        : fetch_(std::move(fetch)), geom_(geom), names_(comp_names), path_(std::move(path)),
          interval_(export_interval) {}

    void exportIfNecessary(int step, amrex::Real time) const {
        if (interval_ <= 0 || step % interval_ != 0) return;
        ScopedTimer timer("PlotExporter::exportIfNecessary()");
        const amrex::Box& dom = geom_.Domain();
        const long long ncell = (long long)dom.length(0) * dom.length(1) * dom.length(2);
        std::vector<double> host(std::size_t(ncell) * names_.size());
        fetch_(host.data());
        write_single_level_plotfile(amrex::Concatenate(path_.string(), step, 5), host.data(), geom_, names_, time,
                                    step);
    }

  private:
    std::function<void(double*)> fetch_;
    amrex::Geometry geom_;
    amrex::Vector<std::string> names_;
    fs::path path_;
    int interval_;
};

} // namespace treesap
