// treesap-b200: periodic export of the state (API of the reference util/PlotExporter.hpp:29-67:
// exportIfNecessary(step, time) writes at step % interval == 0, named path + step zero-padded to 5).
//
// The reference writes AMReX plotfiles through amrex::WriteSingleLevelPlotfile. This build has
// no AMReX; each export is a directory <path><step> holding `Header` (text: component names,
// extents, time, step, geometry) and `data.bin` (FP64 valid cells, [comp][z][y][x]), copied
// from the device after the stream reaches the export point.
#pragma once

#include <AMReX.H>
#include <cuda_runtime.h>

#include <filesystem>
#include <fstream>
#include <functional>
#include <string>
#include <vector>

#include "ScopedTimer.hpp"

namespace treesap {

namespace fs = std::filesystem;

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
        const fs::path dir = amrex::Concatenate(path_.string(), step, 5);
        fs::create_directories(dir);
        std::ofstream h(dir / "Header");
        h << "treesap-b200-plot-1\n" << names_.size() << "\n";
        for (const auto& n : names_) h << n << "\n";
        h << dom.length(0) << " " << dom.length(1) << " " << dom.length(2) << "\n";
        h.precision(17);
        h << time << "\n" << step << "\n";
        for (int d = 0; d < 3; ++d) h << geom_.ProbLo(d) << " " << geom_.ProbHi(d) << " " << geom_.CellSize(d) << "\n";
        std::ofstream b(dir / "data.bin", std::ios::binary);
        b.write(reinterpret_cast<const char*>(host.data()), std::streamsize(host.size() * sizeof(double)));
    }

  private:
    std::function<void(double*)> fetch_;
    amrex::Geometry geom_;
    amrex::Vector<std::string> names_;
    fs::path path_;
    int interval_;
};

} // namespace treesap
