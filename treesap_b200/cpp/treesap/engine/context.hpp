// treesap-b200 engine: host-side access to the runtime of the C ABI (context, stream,
// device error word, TMA descriptors) for the header-only front end.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>

#include <treesap_b200.h>

#include "field.hpp"

namespace treesap_b200 {

inline void ts_check(ts_status s, ts_context* ctx, const char* what) {
    if (s != TS_OK) {
        std::string msg = std::string(what) + ": " + ts_status_string(s);
        if (ctx) msg += std::string(" (") + ts_context_last_error(ctx) + ")";
        throw std::runtime_error(msg);
    }
}

/// Process-wide context of the current device (created on first use, kept until exit).
inline ts_context* default_context() {
    static std::mutex m;
    static std::map<int, ts_context*> per_device;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(m);
    auto it = per_device.find(dev);
    if (it != per_device.end()) return it->second;
    ts_context* ctx = nullptr;
    ts_check(ts_context_create(dev, &ctx), nullptr, "ts_context_create");
    per_device[dev] = ctx;
    return ctx;
}

/// Cache of TMA descriptors, keyed by (device pointer, box, extents, element type).
class TensorMapCache {
  public:
    const CUtensorMap& get(const void* base, const Layout& L, int dtype, int box_x, int box_y) {
        auto key = std::make_tuple(base, box_x, box_y, L.px, L.py, L.pz, dtype);
        auto it = maps_.find(key);
        if (it != maps_.end()) return it->second;
        CUtensorMap m;
        const ts_field_layout cl = L.to_c(dtype);
        ts_check(ts_field_tensor_map(&cl, base, box_x, box_y, &m), nullptr, "ts_field_tensor_map");
        return maps_.emplace(key, m).first->second;
    }
    void clear() { maps_.clear(); }

  private:
    std::map<std::tuple<const void*, int, int, long long, long long, long long, int>, CUtensorMap> maps_;
};

} // namespace treesap_b200
