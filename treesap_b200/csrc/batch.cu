// treesap-b200 C ABI: batched instances (ts_batch_*). See include/treesap_b200.h.
#include <cuda_runtime.h>

#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch_adapter.cuh"
#include "runtime_internal.hpp"

struct ts_batch {
    ts_context* ctx = nullptr;
    treesap_b200::BatchIface* impl = nullptr;
    double* tables = nullptr; // kBatchTableCap doubles per instance (device)
    int count = 0;
};

using namespace treesap_b200;

namespace {

ts_status guarded(ts_context* ctx, const char* what, auto&& fn) {
    try {
        fn();
        return TS_OK;
    } catch (const std::invalid_argument& e) {
        set_error(ctx, std::string(what) + ": " + e.what());
        return TS_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        set_error(ctx, std::string(what) + ": " + e.what());
        const std::string m = e.what();
        return m.find("out of memory") != std::string::npos ? TS_ERR_OUT_OF_MEMORY : TS_ERR_CUDA;
    }
}

/// Every instance: a valid scalar-wave descriptor; all instances share the model type
/// (ngrow, precision, with or without Kreiss-Oliger) and the scheme RK4.
ts_status validate_batch(const ts_wave_desc* d, int count) {
    if (!d || count < 1) return TS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < count; ++i) {
        const ts_wave_desc& e = d[i];
        for (int q = 0; q < 3; ++q) {
            if (e.n[q] < e.ngrow || e.n[q] < 1 || e.n[q] > (1 << 16)) return TS_ERR_INVALID_ARGUMENT;
            if (!(e.prob_hi[q] > e.prob_lo[q])) return TS_ERR_INVALID_ARGUMENT;
        }
        if (!(e.dt > 0.0) || e.ko_strength < 0.0 || e.abl_thickness < 0) return TS_ERR_INVALID_ARGUMENT;
        if (e.precision != TS_PRECISION_F64 && e.precision != TS_PRECISION_F32_STAGE) return TS_ERR_INVALID_ARGUMENT;
        if (e.bc != TS_BC_NOOP && e.bc != TS_BC_DIRICHLET) return TS_ERR_INVALID_ARGUMENT;
        if (e.model != TS_MODEL_WAVE || e.scheme != TS_RK4 || (e.ngrow != 2 && e.ngrow != 4) ||
            e.abl_thickness > 0 || e.c2)
            return TS_ERR_UNSUPPORTED;
        if (e.ngrow != d[0].ngrow || e.precision != d[0].precision || (e.ko_strength > 0.0) != (d[0].ko_strength > 0.0))
            return TS_ERR_INVALID_ARGUMENT;
    }
    return TS_OK;
}

bool valid_instance(const ts_batch* b, int i) { return b && b->impl && i >= 0 && i < b->count; }

} // namespace

extern "C" {

ts_status ts_batch_create(ts_context* ctx, const ts_wave_desc* descs, int count, ts_batch** out) {
    if (!ctx || !out) return TS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    ts_status st = validate_batch(descs, count);
    if (st != TS_OK) {
        set_error(ctx, "ts_batch_create: invalid or unsupported descriptors");
        return st;
    }
    auto* b = new ts_batch();
    b->ctx = ctx;
    b->count = count;
    st = guarded(ctx, "ts_batch_create", [&] {
        const size_t n = kBatchTableCap * size_t(count);
        cuda_check(cudaMalloc(&b->tables, sizeof(double) * n), "cudaMalloc(init tables)");
        cuda_check(cudaMemset(b->tables, 0, sizeof(double) * n), "cudaMemset(init tables)");
        b->impl = descs[0].ngrow == 2 ? make_batch_g2(ctx, descs, count, b->tables)
                                      : make_batch_g4(ctx, descs, count, b->tables);
    });
    if (st != TS_OK) {
        ts_batch_destroy(b);
        return st;
    }
    *out = b;
    return TS_OK;
}

ts_status ts_batch_destroy(ts_batch* b) {
    if (!b) return TS_OK;
    if (b->impl) cudaStreamSynchronize(b->impl->stream());
    delete b->impl;
    if (b->tables) cudaFree(b->tables);
    delete b;
    return TS_OK;
}

int ts_batch_size(const ts_batch* b) { return b ? b->count : 0; }

ts_status ts_batch_initialise(ts_batch* b, int instance, int init_kind, int nitems, const double* items) {
    if (!valid_instance(b, instance)) return TS_ERR_INVALID_ARGUMENT;
    if ((init_kind != TS_INIT_GAUSSIAN && init_kind != TS_INIT_FOURIER) || nitems < 0 || (nitems > 0 && !items) ||
        size_t(2 + 6 * nitems) > kBatchTableCap)
        return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_initialise", [&] {
        std::vector<double> host(2 + 6 * size_t(nitems));
        host[0] = init_kind;
        host[1] = nitems;
        for (int q = 0; q < 6 * nitems; ++q) host[2 + q] = items[q];
        cudaStream_t s = b->impl->stream();
        cuda_check(cudaMemcpyAsync(b->tables + instance * kBatchTableCap, host.data(), host.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, s),
                   "cudaMemcpyAsync(init table)");
        b->impl->initialise(instance);
        cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize(initialise)");
    });
}

ts_status ts_batch_set_state(ts_batch* b, int instance, const double* src, int src_is_device) {
    if (!valid_instance(b, instance) || !src) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_set_state", [&] { b->impl->set_state(instance, src, src_is_device != 0); });
}

ts_status ts_batch_get_state(ts_batch* b, int instance, double* dst, int dst_is_device) {
    if (!valid_instance(b, instance) || !dst) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_get_state", [&] { b->impl->get_state(instance, dst, dst_is_device != 0); });
}

ts_status ts_batch_step(ts_batch* b, int nsteps) {
    if (!b || !b->impl || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_step", [&] { b->impl->step(nsteps); });
}

ts_status ts_batch_use_graph(ts_batch* b, int enable) {
    if (!b || !b->impl) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_use_graph", [&] { b->impl->use_graph(enable != 0); });
}

ts_status ts_batch_set_launch_shape(ts_batch* b, int rows, int zchunk) {
    if (!b || !b->impl || rows < 0 || zchunk < 0) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_set_launch_shape", [&] { b->impl->set_launch_shape(rows, zchunk); });
}

ts_status ts_batch_autotune(ts_batch* b, int trial_steps, int* rows, int* zchunk) {
    if (!b || !b->impl || trial_steps < 1) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_autotune", [&] {
        const auto best = b->impl->autotune(trial_steps);
        if (rows) *rows = best.first;
        if (zchunk) *zchunk = best.second;
    });
}

ts_status ts_batch_last_step_timing(ts_batch* b, double* ms, long long* launches) {
    if (!b || !b->impl) return TS_ERR_INVALID_ARGUMENT;
    return guarded(b->ctx, "ts_batch_last_step_timing", [&] {
        const auto t = b->impl->last_step_timing();
        if (ms) *ms = t.first;
        if (launches) *launches = t.second;
    });
}

} // extern "C"
