// treesap-b200 C ABI: ts_integrator_* entry points (include/treesap_b200.h).
#include <cuda_runtime.h>

#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>

#include "integrator_adapter.cuh"
#include "runtime_internal.hpp"

struct ts_integrator {
    ts_context* ctx = nullptr;
    treesap_b200::IntegratorIface* impl = nullptr;
    double* table = nullptr; // initial-condition parameters (device)
    double* c2 = nullptr;    // c(x)^2 (device) or nullptr
    double* host_stage = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long last_launches = 0;
    // CUDA graphs of one step, for the two buffer parities (state and stage buffers swap every step)
    bool use_graph = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    long long graph_launches[2] = {0, 0}; // kernels in each captured step
    double graph_dt = 0.0;
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

ts_status validate(const ts_wave_desc* d) {
    if (!d) return TS_ERR_INVALID_ARGUMENT;
    if (d->ngrow < 1 || d->ngrow > 4) return TS_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q) {
        if (d->n[q] < d->ngrow || d->n[q] < 1 || d->n[q] > (1 << 16)) return TS_ERR_INVALID_ARGUMENT;
        if (!(d->prob_hi[q] > d->prob_lo[q])) return TS_ERR_INVALID_ARGUMENT;
    }
    if (!(d->dt > 0.0)) return TS_ERR_INVALID_ARGUMENT;
    for (int q = 0; q < 3; ++q)
        if (d->block[q] < 0) return TS_ERR_INVALID_ARGUMENT;
    if (d->model != TS_MODEL_WAVE && d->model != TS_MODEL_TENSOR_WAVE) return TS_ERR_INVALID_ARGUMENT;
    if (d->scheme != TS_EULER && d->scheme != TS_RK4 && d->scheme != TS_DOPRI5) return TS_ERR_INVALID_ARGUMENT;
    if (d->rtol < 0.0 || d->atol < 0.0) return TS_ERR_INVALID_ARGUMENT;
    if (d->precision != TS_PRECISION_F64 && d->precision != TS_PRECISION_F32_STAGE) return TS_ERR_INVALID_ARGUMENT;
    if (d->precision == TS_PRECISION_F32_STAGE && d->scheme != TS_RK4) return TS_ERR_UNSUPPORTED;
    if (d->abl_thickness < 0 || (d->abl_thickness > 0 && d->abl_profile != 1 && d->abl_profile != 2))
        return TS_ERR_INVALID_ARGUMENT;
    // the tensor model is built in its benchmark configuration only (models_tensor_*.cu)
    if (d->model == TS_MODEL_TENSOR_WAVE && (d->ngrow != 3 || d->c2 || d->abl_thickness > 0 || !(d->ko_strength > 0.0) ||
                                             d->bc != TS_BC_NOOP || d->scheme != TS_RK4))
        return TS_ERR_UNSUPPORTED;
    return TS_OK;
}

void drop_graphs(ts_integrator* it) {
    for (auto& g : it->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

cudaStream_t stream_of(ts_integrator* it) { return static_cast<cudaStream_t>(ts_context_stream(it->ctx)); }

SlabOps* slab_of(ts_integrator* it) { return it && it->impl ? it->impl->slab_ops() : nullptr; }

} // namespace

extern "C" {

ts_status ts_integrator_create(ts_context* ctx, const ts_wave_desc* desc, ts_integrator** out) {
    if (!ctx || !out) return TS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    ts_status st = validate(desc);
    if (st != TS_OK) {
        set_error(ctx, "ts_integrator_create: invalid or unsupported descriptor");
        return st;
    }
    auto* it = new ts_integrator();
    it->ctx = ctx;
    st = guarded(ctx, "ts_integrator_create", [&] {
        cuda_check(cudaMalloc(&it->table, sizeof(double) * kInitTableCap), "cudaMalloc(init table)");
        cuda_check(cudaMemset(it->table, 0, sizeof(double) * kInitTableCap), "cudaMemset(init table)");
        if (desc->c2) {
            const size_t n = size_t(desc->n[0]) * desc->n[1] * desc->n[2];
            cuda_check(cudaMalloc(&it->c2, n * sizeof(double)), "cudaMalloc(c2)");
            cuda_check(cudaMemcpy(it->c2, desc->c2, n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(c2)");
        }
        cuda_check(cudaEventCreate(&it->ev0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&it->ev1), "cudaEventCreate");
        if (desc->model == TS_MODEL_TENSOR_WAVE) {
            it->impl = desc->precision == TS_PRECISION_F32_STAGE ? make_tensor_f32(ctx, *desc, it->table)
                                                                 : make_tensor_f64(ctx, *desc, it->table);
        } else {
            switch (desc->ngrow) {
            case 1: it->impl = make_wave_g1(ctx, *desc, it->table, it->c2); break;
            case 2: it->impl = make_wave_g2(ctx, *desc, it->table, it->c2); break;
            case 3: it->impl = make_wave_g3(ctx, *desc, it->table, it->c2); break;
            case 4: it->impl = make_wave_g4(ctx, *desc, it->table, it->c2); break;
            }
        }
        it->graph_dt = desc->dt;
    });
    if (st != TS_OK) {
        ts_integrator_destroy(it);
        return st;
    }
    *out = it;
    return TS_OK;
}

ts_status ts_integrator_create_slab(ts_context* ctx, const ts_wave_desc* desc, int zlo, int nz, int lo_ex, int hi_ex,
                                    ts_integrator** out) {
    if (!ctx || !out || !desc) return TS_ERR_INVALID_ARGUMENT;
    if (zlo < 0 || nz < desc->ngrow || zlo + nz > desc->n[2] || desc->c2 || desc->model != TS_MODEL_WAVE) {
        set_error(ctx, "ts_integrator_create_slab: slab outside the domain, thinner than the ghost width, or a model "
                       "without slab support");
        return TS_ERR_INVALID_ARGUMENT;
    }
    SlabRequest& r = slab_request();
    r.active = true;
    r.sz.zoff = zlo;
    r.sz.nz = desc->n[2];
    r.sz.lo_ex = lo_ex != 0;
    r.sz.hi_ex = hi_ex != 0;
    r.depth = nz;
    const ts_status st = ts_integrator_create(ctx, desc, out);
    r = SlabRequest{};
    return st;
}

int ts_slab_stages(ts_integrator* it) {
    SlabOps* s = slab_of(it);
    return s ? s->stages() : 0;
}

ts_status ts_slab_prepare(ts_integrator* it, int stage) {
    SlabOps* s = slab_of(it);
    if (!s || stage < 0 || stage >= s->stages()) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_prepare", [&] { s->prepare(stage); });
}

ts_status ts_slab_send_planes(ts_integrator* it, int stage, int face, void** ptr, long long* elems,
                              long long* comp_stride, int* elem_size) {
    SlabOps* s = slab_of(it);
    if (!s || stage < 0 || stage >= s->stages() || (face != 0 && face != 1) || !ptr || !elems || !comp_stride ||
        !elem_size)
        return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_send_planes",
                   [&] { s->send_planes(stage, face, ptr, elems, comp_stride, elem_size); });
}

ts_status ts_slab_receive_planes(ts_integrator* it, int stage, int face, const void* buf) {
    SlabOps* s = slab_of(it);
    if (!s || stage < 0 || stage >= s->stages() || (face != 0 && face != 1) || !buf) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_receive_planes", [&] { s->receive_planes(stage, face, buf); });
}

ts_status ts_slab_fill(ts_integrator* it, int stage) {
    SlabOps* s = slab_of(it);
    if (!s || stage < 0 || stage >= s->stages()) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_fill", [&] { s->fill(stage); });
}

ts_status ts_slab_launch(ts_integrator* it, int stage) {
    SlabOps* s = slab_of(it);
    if (!s || stage < 0 || stage >= s->stages()) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_launch", [&] { s->launch(stage); });
}

ts_status ts_slab_finish(ts_integrator* it) {
    SlabOps* s = slab_of(it);
    if (!s) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_slab_finish", [&] { s->finish(); });
}

ts_status ts_integrator_destroy(ts_integrator* it) {
    if (!it) return TS_OK;
    if (it->ctx) cudaStreamSynchronize(stream_of(it));
    drop_graphs(it);
    delete it->impl;
    if (it->table) cudaFree(it->table);
    if (it->c2) cudaFree(it->c2);
    if (it->ev0) cudaEventDestroy(it->ev0);
    if (it->ev1) cudaEventDestroy(it->ev1);
    delete it;
    return TS_OK;
}

int ts_integrator_ncomp(const ts_integrator* it) { return (it && it->impl) ? it->impl->ncomp() : 0; }

ts_status ts_integrator_initialise(ts_integrator* it, int init_kind, int nitems, const double* items) {
    if (!it || !it->impl) return TS_ERR_INVALID_ARGUMENT;
    if ((init_kind != TS_INIT_GAUSSIAN && init_kind != TS_INIT_FOURIER) || nitems < 0 || (nitems > 0 && !items))
        return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_initialise", [&] { it->impl->initialise(init_kind, nitems, items); });
}

ts_status ts_integrator_initialise_expressions(ts_integrator* it, int count, const char* const* exprs) {
    if (!it || !it->impl || !exprs || count < 1) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_initialise_expressions",
                   [&] { it->impl->initialise_expressions(count, exprs); });
}

ts_status ts_expression_eval(const char* expr, int n, const double* x, const double* y, const double* z,
                             double* out) {
    if (!expr || n < 0 || (n > 0 && (!x || !y || !z || !out))) return TS_ERR_INVALID_ARGUMENT;
    try {
        const std::vector<treesap::expr::Instr> code = treesap::expr::Compiler::compile(expr);
        for (int q = 0; q < n; ++q) out[q] = treesap::expr::eval(code.data(), int(code.size()), x[q], y[q], z[q]);
    } catch (const std::exception&) {
        return TS_ERR_INVALID_ARGUMENT;
    }
    return TS_OK;
}

ts_status ts_integrator_set_state(ts_integrator* it, const double* src, int src_is_device) {
    if (!it || !it->impl || !src) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_set_state", [&] { it->impl->set_state(src, src_is_device != 0); });
}

ts_status ts_integrator_get_state(ts_integrator* it, double* dst, int dst_is_device) {
    if (!it || !it->impl || !dst) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_get_state", [&] { it->impl->get_state(dst, dst_is_device != 0); });
}

ts_status ts_integrator_adaptive_stats(ts_integrator* it, long long* accepted, long long* rejected, double* next_dt,
                                       double* last_error) {
    if (!it || !it->impl || !accepted || !rejected || !next_dt || !last_error) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_adaptive_stats",
                   [&] { it->impl->adaptive_stats(accepted, rejected, next_dt, last_error); });
}

ts_status ts_integrator_check_finite(ts_integrator* it) {
    if (!it || !it->impl) return TS_ERR_INVALID_ARGUMENT;
    bool finite = true;
    const ts_status st = guarded(it->ctx, "ts_integrator_check_finite", [&] { finite = it->impl->state_is_finite(); });
    if (st != TS_OK) return st;
    if (!finite) {
        set_error(it->ctx, "ts_integrator_check_finite: the state holds NaN or infinite values");
        return TS_ERR_NONFINITE;
    }
    return TS_OK;
}

ts_status ts_integrator_step(ts_integrator* it, int nsteps) {
    if (!it || !it->impl || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_step", [&] {
        cudaStream_t s = stream_of(it);
        cuda_check(cudaEventRecord(it->ev0, s), "cudaEventRecord");
        long long launches = 0;
        for (int q = 0; q < nsteps; ++q) {
            if (it->use_graph) {
                const int parity = int(it->impl->steps() & 1);
                if (!it->graph[parity]) {
                    // capture this step (the built-in models are autonomous with time-independent
                    // boundary data, so replays with the captured stage times are exact)
                    cudaGraph_t g;
                    cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
                    try {
                        it->impl->step();
                    } catch (...) {
                        cudaStreamEndCapture(s, &g);
                        throw;
                    }
                    cuda_check(cudaStreamEndCapture(s, &g), "cudaStreamEndCapture");
                    cuda_check(cudaGraphInstantiate(&it->graph[parity], g, 0), "cudaGraphInstantiate");
                    cudaGraphDestroy(g);
                    it->graph_launches[parity] = it->impl->launches_per_step();
                    // the capture ran the host bookkeeping (swaps, clock) but no device work: launch it once
                    cuda_check(cudaGraphLaunch(it->graph[parity], s), "cudaGraphLaunch");
                } else {
                    cuda_check(cudaGraphLaunch(it->graph[parity], s), "cudaGraphLaunch");
                    it->impl->step_host_only();
                }
                launches += it->graph_launches[parity];
            } else {
                it->impl->step();
                launches += it->impl->launches_per_step();
            }
        }
        cuda_check(cudaEventRecord(it->ev1, s), "cudaEventRecord");
        it->last_launches = launches;
    });
}

ts_status ts_integrator_run(ts_integrator* it, const double* host_in, int nsteps, double* host_out) {
    if (!it || !it->impl || !host_in || !host_out || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    ts_status st = ts_integrator_set_state(it, host_in, 0);
    if (st == TS_OK) st = ts_integrator_step(it, nsteps);
    if (st == TS_OK) st = ts_integrator_get_state(it, host_out, 0);
    if (st == TS_OK) st = ts_context_sync(it->ctx);
    return st;
}

ts_status ts_integrator_time(const ts_integrator* it, double* time, long long* steps) {
    if (!it || !it->impl) return TS_ERR_INVALID_ARGUMENT;
    if (time) *time = it->impl->time();
    if (steps) *steps = it->impl->steps();
    return TS_OK;
}

ts_status ts_integrator_state_field(ts_integrator* it, void** device_ptr, ts_field_layout* layout) {
    if (!it || !it->impl) return TS_ERR_INVALID_ARGUMENT;
    if (device_ptr) *device_ptr = it->impl->state_ptr();
    if (layout) *layout = it->impl->state_layout().to_c(TS_F64);
    return TS_OK;
}

ts_status ts_integrator_use_graph(ts_integrator* it, int enable) {
    if (!it || !it->impl) return TS_ERR_INVALID_ARGUMENT;
    cudaStreamSynchronize(stream_of(it));
    drop_graphs(it);
    it->use_graph = enable != 0;
    return TS_OK;
}

ts_status ts_integrator_profile(ts_integrator* it, int nsteps, int nclasses, long long* launches, double* ms) {
    if (!it || !it->impl || nsteps < 0 || nclasses < 1 || !launches || !ms) return TS_ERR_INVALID_ARGUMENT;
    return guarded(it->ctx, "ts_integrator_profile", [&] {
        treesap::KernelClock clock;
        it->impl->attach_clock(&clock);
        try {
            for (int q = 0; q < nsteps; ++q) it->impl->step();
        } catch (...) {
            it->impl->attach_clock(nullptr);
            throw;
        }
        it->impl->attach_clock(nullptr);
        cuda_check(cudaStreamSynchronize(stream_of(it)), "cudaStreamSynchronize");
        clock.collect(nclasses, launches, ms);
    });
}

ts_status ts_integrator_set_launch_shape(ts_integrator* it, int rows, int chunks) {
    if (!it || !it->impl || rows < 0 || chunks < 0) return TS_ERR_INVALID_ARGUMENT;
    drop_graphs(it);
    it->impl->set_launch_shape(rows, chunks);
    return TS_OK;
}

ts_status ts_integrator_last_step_timing(ts_integrator* it, double* ms, long long* launches) {
    if (!it) return TS_ERR_INVALID_ARGUMENT;
    float f = 0.f;
    cudaError_t e = cudaEventElapsedTime(&f, it->ev0, it->ev1);
    if (e != cudaSuccess) return from_cuda(it->ctx, e, "cudaEventElapsedTime");
    if (ms) *ms = f;
    if (launches) *launches = it->last_launches;
    return TS_OK;
}

} // extern "C"
