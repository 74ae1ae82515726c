// treesap-b200 C ABI: helpers shared by the library's translation units (not installed).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include <treesap_b200.h>

#include "../cpp/treesap/engine/field.hpp"
#include "../cpp/treesap/engine/ptx.cuh"

namespace treesap_b200 {
void set_error(ts_context* ctx, const std::string& msg);
ts_status from_cuda(ts_context* ctx, cudaError_t e, const char* what);
} // namespace treesap_b200
