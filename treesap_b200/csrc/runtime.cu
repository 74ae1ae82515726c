// treesap-b200 C ABI: runtime services (contexts, field layouts, TMA descriptors).
// See include/treesap_b200.h for the contract of every entry point.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <treesap_b200.h>

#include "runtime_internal.hpp"

struct ts_context {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    int* err = nullptr;      // device error word
    int* err_host = nullptr; // pinned mirror
    std::string last_error;
    // pending TS_FAULT_SKIP_COPY (plane < 0: none), taken by the next stage launch
    std::mutex fault_mutex;
    int fault_plane = -1;
};

namespace treesap_b200 {

void set_error(ts_context* ctx, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
}

ts_status from_cuda(ts_context* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TS_OK;
    (void)cudaGetLastError(); // clear the last-error slot so later launch checks do not repeat it
    set_error(ctx, std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}
} // namespace
} // namespace treesap_b200

using namespace treesap_b200;

extern "C" {

int ts_abi_version(void) { return TS_ABI_VERSION; }

const char* ts_status_string(ts_status s) {
    switch (s) {
    case TS_OK: return "TS_OK";
    case TS_ERR_INVALID_ARGUMENT: return "TS_ERR_INVALID_ARGUMENT";
    case TS_ERR_UNSUPPORTED: return "TS_ERR_UNSUPPORTED";
    case TS_ERR_CUDA: return "TS_ERR_CUDA";
    case TS_ERR_OUT_OF_MEMORY: return "TS_ERR_OUT_OF_MEMORY";
    case TS_ERR_DEVICE: return "TS_ERR_DEVICE";
    case TS_ERR_NO_DEVICE: return "TS_ERR_NO_DEVICE";
    case TS_ERR_NONFINITE: return "TS_ERR_NONFINITE";
    }
    return "TS_ERR_UNKNOWN";
}

ts_status ts_context_create(int device, ts_context** out) {
    if (!out) return TS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return TS_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return TS_ERR_INVALID_ARGUMENT;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TS_ERR_CUDA;
    if (prop.major != 10) return TS_ERR_NO_DEVICE; // built for sm_100a only
    auto* ctx = new ts_context();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ts_status st = TS_OK;
    if ((st = from_cuda(ctx, cudaSetDevice(device), "cudaSetDevice")) == TS_OK &&
        (st = from_cuda(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ==
            TS_OK &&
        (st = from_cuda(ctx, cudaMalloc(&ctx->err, sizeof(int)), "cudaMalloc(error word)")) == TS_OK &&
        (st = from_cuda(ctx, cudaMemset(ctx->err, 0, sizeof(int)), "cudaMemset(error word)")) == TS_OK &&
        (st = from_cuda(ctx, cudaMallocHost(&ctx->err_host, sizeof(int)), "cudaMallocHost")) == TS_OK) {
        *out = ctx;
        return TS_OK;
    }
    ts_context_destroy(ctx);
    return st;
}

ts_status ts_context_destroy(ts_context* ctx) {
    if (!ctx) return TS_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->err) cudaFree(ctx->err);
    if (ctx->err_host) cudaFreeHost(ctx->err_host);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    cudaSetDevice(cur);
    delete ctx;
    return TS_OK;
}

ts_status ts_context_sync(ts_context* ctx) {
    if (!ctx) return TS_ERR_INVALID_ARGUMENT;
    ts_status st = from_cuda(ctx, cudaMemcpyAsync(ctx->err_host, ctx->err, sizeof(int), cudaMemcpyDeviceToHost,
                                                  ctx->stream),
                             "cudaMemcpyAsync(error word)");
    if (st != TS_OK) return st;
    if ((st = from_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize")) != TS_OK) return st;
    const int word = *ctx->err_host;
    if (word != 0) {
        cudaMemsetAsync(ctx->err, 0, sizeof(int), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        char buf[160];
        std::snprintf(buf, sizeof buf, "device error word 0x%x (%s%s%s)", word,
                      (word & kErrMbarTimeout) ? "mbarrier wait timed out " : "",
                      (word & kErrBounds) ? "index out of bounds " : "",
                      (word & kErrBadLaunch) ? "inconsistent launch" : "");
        set_error(ctx, buf);
        return TS_ERR_DEVICE;
    }
    return TS_OK;
}

ts_status ts_context_inject_fault(ts_context* ctx, int fault, long long arg) {
    if (!ctx) return TS_ERR_INVALID_ARGUMENT;
    switch (fault) {
    case TS_FAULT_NONE: {
        std::lock_guard<std::mutex> lock(ctx->fault_mutex);
        ctx->fault_plane = -1;
        alloc_faults() = 0;
        return TS_OK;
    }
    case TS_FAULT_SKIP_COPY: {
        if (arg < 0 || arg > (1 << 20)) return TS_ERR_INVALID_ARGUMENT;
        std::lock_guard<std::mutex> lock(ctx->fault_mutex);
        ctx->fault_plane = int(arg);
        return TS_OK;
    }
    case TS_FAULT_ALLOC:
        if (arg < 0 || arg > (1 << 20)) return TS_ERR_INVALID_ARGUMENT;
        alloc_faults() = int(arg);
        return TS_OK;
    default: return TS_ERR_INVALID_ARGUMENT;
    }
}

int ts_context_take_stage_fault(ts_context* ctx, int* plane, unsigned long long* wait_ns) {
    if (!ctx || !plane || !wait_ns) return 0;
    std::lock_guard<std::mutex> lock(ctx->fault_mutex);
    if (ctx->fault_plane < 0) return 0;
    *plane = ctx->fault_plane;
    *wait_ns = kInjectedWaitLimitNs;
    ctx->fault_plane = -1;
    return 1;
}

const char* ts_context_last_error(const ts_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }
void* ts_context_stream(ts_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }
int* ts_context_error_word(ts_context* ctx) { return ctx ? ctx->err : nullptr; }
int ts_context_sm_count(const ts_context* ctx) { return ctx ? ctx->sm_count : 0; }

ts_status ts_field_layout_make(const int n[3], int ngrow, int ncomp, int dtype, ts_field_layout* out) {
    if (!n || !out || ngrow < 0 || ngrow > 8 || ncomp < 1 || (dtype != TS_F64 && dtype != TS_F32))
        return TS_ERR_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d)
        if (n[d] < 1 || n[d] < ngrow) return TS_ERR_INVALID_ARGUMENT;
    if (!Layout::rows_fit(n, ngrow)) return TS_ERR_INVALID_ARGUMENT;
    const Layout L = Layout::make(n, ngrow, ncomp, dtype == TS_F64 ? 8 : 4);
    *out = L.to_c(dtype);
    return TS_OK;
}

long long ts_field_bytes(const ts_field_layout* l) {
    if (!l) return 0;
    return l->px * l->py * l->pz * l->ncomp * (l->dtype == TS_F64 ? 8 : 4);
}

ts_status ts_field_tensor_map(const ts_field_layout* l, const void* base, int box_x, int box_y, void* out) {
    if (!l || !base || !out || box_x < 1 || box_x > 256 || box_y < 1 || box_y > 256 || l->ncomp > 256)
        return TS_ERR_INVALID_ARGUMENT;
    const int es = (l->dtype == TS_F64) ? 8 : 4;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (box_x * es) % 16 != 0 || (l->px * es) % 16 != 0)
        return TS_ERR_INVALID_ARGUMENT;
    auto enc = encode_fn();
    if (!enc) return TS_ERR_CUDA;
    const cuuint64_t dims[4] = {cuuint64_t(l->px), cuuint64_t(l->py), cuuint64_t(l->pz), cuuint64_t(l->ncomp)};
    const cuuint64_t strides[3] = {cuuint64_t(l->px * es), cuuint64_t(l->px * l->py * es),
                                   cuuint64_t(l->px * l->py * l->pz * es)};
    const cuuint32_t box[4] = {cuuint32_t(box_x), cuuint32_t(box_y), 1u, cuuint32_t(l->ncomp)};
    const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
    CUresult r = enc(reinterpret_cast<CUtensorMap*>(out),
                     l->dtype == TS_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                     const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? TS_OK : TS_ERR_CUDA;
}

} // extern "C"
