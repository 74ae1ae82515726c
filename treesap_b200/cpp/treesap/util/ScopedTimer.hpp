// treesap-b200: RAII host wall-clock scope timers with per-name totals, mean and standard
// deviation (API of the reference util/ScopedTimer.hpp:34-149: ScopedTimer(name),
// static printOverview(), static bool enabled, off by default). Like the reference, the
// timers do not synchronise the device: around asynchronous integrator calls they measure
// host-side enqueue time. Device times come from CUDA events (ts_integrator_last_step_timing).
#pragma once

#include <AMReX.H>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace treesap {

class ScopedTimer {
    using Clock = std::chrono::steady_clock;

    struct Stats {
        double total_us = 0.0;
        double sum_sq_us = 0.0;
        std::size_t count = 0;
        double mean() const { return count ? total_us / double(count) : 0.0; }
        double stdev() const {
            if (!count) return 0.0;
            const double m = mean(), v = sum_sq_us / double(count) - m * m;
            return v > 0.0 ? std::sqrt(v) : 0.0;
        }
    };

  public:
    explicit ScopedTimer(std::string name) : name_(std::move(name)), start_(Clock::now()) {}

    ~ScopedTimer() {
        if (!enabled) return;
        const double us = std::chrono::duration<double, std::micro>(Clock::now() - start_).count();
        Stats& s = table()[name_];
        s.total_us += us;
        s.sum_sq_us += us * us;
        ++s.count;
        amrex::AllPrint() << "[Timer: " << name_ << "] Run: " << format(us) << " | Total: " << format(s.total_us)
                          << " | Avg: " << format(s.mean()) << " | StdDev: " << format(s.stdev()) << " (" << s.count
                          << " runs)\n";
    }

    /// Table of all timers so far, sorted by total time.
    static void printOverview() {
        amrex::AllPrint() << "--- --- --- ScopedTimer Profiling Overview --- --- ---" << std::endl;
        std::vector<std::pair<std::string, Stats>> rows(table().begin(), table().end());
        std::sort(rows.begin(), rows.end(), [](const auto& a, const auto& b) { return a.second.total_us > b.second.total_us; });
        for (const auto& [name, s] : rows) {
            std::cout << "[Timer: " << std::left << std::setw(35) << name << "] " << std::right
                      << "Executions: " << std::setw(6) << s.count << " | Total: " << std::setw(8) << format(s.total_us)
                      << " | Avg: " << std::setw(8) << format(s.mean()) << " | StdDev: " << std::setw(9)
                      << format(s.stdev()) << std::endl;
        }
    }

    inline static bool enabled = false;

  private:
    static std::map<std::string, Stats>& table() {
        static std::map<std::string, Stats> t;
        return t;
    }
    static std::string format(double us) {
        std::ostringstream os;
        os << std::fixed << std::setprecision(1);
        if (us < 1000.0)
            os << us << " µs";
        else if (us < 1e6)
            os << us / 1000.0 << " ms";
        else
            os << us / 1e6 << " s";
        return os.str();
    }

    std::string name_;
    Clock::time_point start_;
};

} // namespace treesap
