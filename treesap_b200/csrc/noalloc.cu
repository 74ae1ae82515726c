// treesap-b200 C ABI: ts_wave_rk4_steps_noalloc, RK4 steps that allocate no device memory.
//
// Some callers cannot call cudaMalloc: host applications that hand all device memory to
// their own pool or arena and forbid outside allocations, and latency-sensitive loops for
// which cudaMalloc/cudaFree are off limits because they may synchronise the whole device
// and stall the caller's other streams. For them this entry point runs the same fused RK4
// stage kernels and ghost fills as ts_integrator_step on a caller-owned state buffer; its
// three RK4 stage registers and its device error word live in one static device array of
// TS_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds until exit.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>

#include "integrator_adapter.cuh"
#include "runtime_internal.hpp"

namespace {

using namespace treesap_b200;

// The scratch array. In host code `scratch` is only a stand-in for the symbol, never a device
// address: the device address comes from cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char scratch[TS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
constexpr size_t kAlign = 256;

/// Device address of `scratch` on the current device, looked up once per device.
ts_status scratch_address(int device, unsigned char** out) {
    static std::mutex m;
    static unsigned char* addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) return TS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(m);
    if (!addr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, scratch) != cudaSuccess || !p) return TS_ERR_CUDA;
        addr[device] = static_cast<unsigned char*>(p);
    }
    *out = addr[device];
    return TS_OK;
}

size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

template <class RHS, class BC>
void run_steps(const ts_wave_desc& d, const RHS& rhs, const BC& bc, double* state, unsigned char* base, int nsteps,
               cudaStream_t stream) {
    constexpr int G = RHS::ngrow, NC = RHS::ncomp;
    using Tile = typename treesap::detail::DefaultTile<double, G, NC>::type;
    const Layout L = Layout::make(d.n, G, NC, sizeof(double));
    const size_t fbytes = round_up(size_t(L.bytes()));
    int* err = reinterpret_cast<int*>(base);
    double* s_new = reinterpret_cast<double*>(base + kAlign);
    double* s_arg = reinterpret_cast<double*>(base + kAlign + fbytes);
    double* s_argn = reinterpret_cast<double*>(base + kAlign + 2 * fbytes);
    // The array keeps the previous call's contents: start from zeroed registers and error word,
    // as freshly allocated integrator buffers do.
    cuda_check(cudaMemsetAsync(base, 0, kAlign + 3 * fbytes, stream), "cudaMemsetAsync(scratch)");

    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    const amrex::GeometryData geom = geometry_of(d).data();

    auto fill = [&](double* f, double t) {
        launch_ghost_fill(f, L, geom, bc, nullptr, t, GhostMode::Functor, sms, stream);
    };
    constexpr double a_frac[4] = {0.0, 0.5, 0.5, 1.0};
    constexpr double b_frac[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    double* old_ = state;
    double* new_ = s_new;
    double* arg = s_arg;
    double* argn = s_argn;
    double time = 0.0;
    const double dt = d.dt;

    auto stage = [&](auto stage_tag, const double* input, double t_arg) {
        constexpr int s = decltype(stage_tag)::value;
        using Launcher = StageLauncher<Tile, RHS, EpiRK4<s>>;
        const auto shape = Launcher::shape(L, sms);
        CUtensorMap tm;
        const ts_field_layout cl = L.to_c(TS_F64);
        if (ts_field_tensor_map(&cl, input, Launcher::box_x(), Launcher::box_y(shape), &tm) != TS_OK)
            throw std::runtime_error("ts_field_tensor_map failed");
        StageParams<double> sp{};
        sp.in = input;
        sp.L = L;
        sp.geom = geom;
        sp.time = t_arg;
        sp.err = err;
        typename EpiRK4<s>::Params ep{new_, argn, old_, L, dt * b_frac[s], dt * a_frac[(s + 1) % 4]};
        CUtensorMap cmap[2];
        int nmap = 0;
        const CentreMaps cm = Launcher::centre_maps(
            [&](const void* b, const Layout& Lc, int dtype, int bx, int by) -> const CUtensorMap& {
                CUtensorMap& m = cmap[nmap++ & 1];
                const ts_field_layout c = Lc.to_c(dtype);
                if (ts_field_tensor_map(&c, b, bx, by, &m) != TS_OK)
                    throw std::runtime_error("ts_field_tensor_map failed");
                return m;
            },
            ep, shape);
        Launcher::launch(tm, cm, sp, rhs, ep, shape, stream);
    };

    for (int n = 0; n < nsteps; ++n) {
        fill(old_, time);
        stage(std::integral_constant<int, 0>{}, old_, time);
        std::swap(arg, argn);
        fill(arg, time + dt * a_frac[1]);
        stage(std::integral_constant<int, 1>{}, arg, time + dt * a_frac[1]);
        std::swap(arg, argn);
        fill(arg, time + dt * a_frac[2]);
        stage(std::integral_constant<int, 2>{}, arg, time + dt * a_frac[2]);
        std::swap(arg, argn);
        fill(arg, time + dt * a_frac[3]);
        stage(std::integral_constant<int, 3>{}, arg, time + dt * a_frac[3]);
        std::swap(old_, new_);
        time += dt;
    }
    if (old_ != state)
        cuda_check(cudaMemcpyAsync(state, old_, size_t(L.bytes()), cudaMemcpyDeviceToDevice, stream),
                   "cudaMemcpyAsync(state)");

    int word = 0;
    cuda_check(cudaMemcpyAsync(&word, err, sizeof(int), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync(error)");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    if (word != 0) throw std::domain_error("device error word set");
}

template <class RHS>
void dispatch_bc(const ts_wave_desc& d, const RHS& rhs, double* state, unsigned char* base, int nsteps,
                 cudaStream_t stream) {
    constexpr int G = RHS::ngrow, NC = RHS::ncomp;
    if (d.bc == TS_BC_DIRICHLET) {
        treesap::DirichletBC<NC, G> bc{};
        for (int c = 0; c < NC; ++c) bc.boundary_values[c] = d.bc_values[c];
        run_steps(d, rhs, bc, state, base, nsteps, stream);
    } else {
        run_steps(d, rhs, treesap::NoOpBC<NC, G>{}, state, base, nsteps, stream);
    }
}

} // namespace

extern "C" ts_status ts_wave_rk4_steps_noalloc(const ts_wave_desc* desc, double* state, int nsteps, void* stream) {
    if (!desc || !state || nsteps < 0) return TS_ERR_INVALID_ARGUMENT;
    const ts_wave_desc& d = *desc;
    if (d.model != TS_MODEL_WAVE || d.ngrow != 2 || d.scheme != TS_RK4 || d.precision != TS_PRECISION_F64 ||
        d.abl_thickness > 0 || d.c2 || d.ko_strength < 0.0 || (d.block[2] > 0 && d.block[2] < d.n[2]))
        return TS_ERR_UNSUPPORTED;
    for (int q = 0; q < 3; ++q)
        if (d.n[q] < d.ngrow || !(d.prob_hi[q] > d.prob_lo[q])) return TS_ERR_INVALID_ARGUMENT;
    if (!(d.dt > 0.0) || (reinterpret_cast<uintptr_t>(state) & 15) != 0) return TS_ERR_INVALID_ARGUMENT;
    // Sizes beyond the static array are rejected before any work is enqueued.
    const Layout L = Layout::make(d.n, 2, 2, sizeof(double));
    if (kAlign + 3 * round_up(size_t(L.bytes())) > size_t(TS_NOALLOC_SCRATCH_BYTES)) return TS_ERR_INVALID_ARGUMENT;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TS_ERR_NO_DEVICE;
    unsigned char* base = nullptr;
    ts_status st = scratch_address(dev, &base);
    if (st != TS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // On an error part-way through, kernels already queued may still write to `state` and to
    // the scratch array: wait for the stream (ignoring its status) before returning, so that
    // no work of this call is in flight once it has returned.
    try {
        if (d.ko_strength > 0.0)
            dispatch_bc(d, treesap::KODecorator<tsb::WaveRHS<2>>{tsb::WaveRHS<2>{}, d.ko_strength}, state, base, nsteps,
                        s);
        else
            dispatch_bc(d, tsb::WaveRHS<2>{}, state, base, nsteps, s);
    } catch (const std::domain_error&) {
        (void)cudaStreamSynchronize(s);
        return TS_ERR_DEVICE;
    } catch (const std::exception&) {
        (void)cudaStreamSynchronize(s);
        return TS_ERR_CUDA;
    }
    return TS_OK;
}
