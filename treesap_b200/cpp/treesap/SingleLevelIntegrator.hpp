// treesap-b200: single-level integrator base (reference SingleLevelIntegrator.hpp:18-188).
//
// Owns the FP64 state (state_old / state_new, ncomp components, ngrow ghost cells) in HBM,
// evaluates the initial condition on the device, fills ghost cells before every step and
// swaps the state after it. Differences from the reference that do not change results:
//   * the domain is one box in HBM; block_size is accepted and validated but the work is
//     decomposed by the stage kernels' tiles instead (the ghost cells that AMReX would
//     exchange between boxes are interior cells here and hold the same values);
//   * all device work runs asynchronously on the context's CUDA stream.
#pragma once

#include <AMReX.H>
#include <cuda_runtime.h>

#include <functional>
#include <optional>
#include <stdexcept>
#include <vector>

#include "Integrator.hpp"
#include "engine/context.hpp"
#include "engine/field.hpp"
#include "engine/grid_kernels.cuh"
#include "engine/stage_kernel.cuh"
#include "pde-model/PDEModelConcepts.hpp"

namespace treesap {

/// Optional per-launch device clock: when attached to an integrator, every kernel launch is
/// bracketed by a CUDA event pair on the integrator's stream and tagged with a class
/// (0 ghost fill, 1 + s for stage s of the step).
struct KernelClock {
    struct Span {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Span> spans;
    void begin(int cls, cudaStream_t s) {
        Span sp{cls, nullptr, nullptr};
        treesap_b200::cuda_check(cudaEventCreate(&sp.a), "cudaEventCreate");
        treesap_b200::cuda_check(cudaEventCreate(&sp.b), "cudaEventCreate");
        treesap_b200::cuda_check(cudaEventRecord(sp.a, s), "cudaEventRecord");
        spans.push_back(sp);
    }
    void end(cudaStream_t s) { treesap_b200::cuda_check(cudaEventRecord(spans.back().b, s), "cudaEventRecord"); }
    /// Sums launch counts and milliseconds per class (after the stream has completed).
    void collect(int nclasses, long long* launches, double* ms) {
        for (int c = 0; c < nclasses; ++c) launches[c] = 0, ms[c] = 0.0;
        for (auto& sp : spans) {
            float f = 0.f;
            cudaEventElapsedTime(&f, sp.a, sp.b);
            if (sp.cls >= 0 && sp.cls < nclasses) {
                launches[sp.cls] += 1;
                ms[sp.cls] += f;
            }
            cudaEventDestroy(sp.a);
            cudaEventDestroy(sp.b);
        }
        spans.clear();
    }
};

namespace detail {
/// Tile shape of the fused stage kernel for a value type, ghost width and component count:
/// CX cells per thread along x, TY rows (consumer warps) plus the producer warp, P planes of
/// prefetch, MINB CTAs per SM, U planes per iteration, CY rows per consumer warp;
/// TREESAP_B200_TILE_F64 / _F32 override the defaults at build time as the decimal number
/// [CY] CX TY(2 digits) P MINB U, e.g. 107222 (CY = 1) or 2105421;
/// when two FP64 centre-operand fields would not fit the shared-memory budget (many
/// components), narrower tiles.
#ifndef TREESAP_B200_TILE_F64
#define TREESAP_B200_TILE_F64 107421
#endif
#ifndef TREESAP_B200_TILE_F32
#define TREESAP_B200_TILE_F32 207421
#endif
// Circular register queue (TileCfg::ROT) for FP64 / FP32 stencil inputs of at most 4
// components: it removes the per-plane queue shift (16 moves per FP64 component and cell at
// ngrow 4) at the price of a plane loop unrolled 2 ngrow + 1 times. Measured at 256^3, ngrow 4:
// FP64 stages 3-10% faster; FP32 stages (two cells per thread) 30% slower, so off for FP32.
// One cell per thread only: with more, the unrolled loop outgrows full unrolling and the queue
// index stops being a compile-time constant (the queue then lands in local memory).
#ifndef TREESAP_B200_QROT_F64
#define TREESAP_B200_QROT_F64 1
#endif
#ifndef TREESAP_B200_QROT_F32
#define TREESAP_B200_QROT_F32 0
#endif
template <int code> struct TileSpec {
    static constexpr int CY = code / 1000000 > 0 ? code / 1000000 : 1, CX = code / 100000 % 10,
                         TY = code / 1000 % 100, P = code / 100 % 10, MINB = code / 10 % 10, U = code % 10;
};
// Models of more than kQueueMaxComponents components stream only the centre planes and read
// their z taps from global memory (TileCfg::ZQ = false): a register queue of 2 ngrow + 1 planes
// of every component does not fit the registers (12 FP64 components at ngrow 3: 168 registers
// of queue alone, kilobytes of spills). Their tiles: TREESAP_B200_TILE_MANY_F64 / _F32.
#ifndef TREESAP_B200_TILE_MANY_F64
#define TREESAP_B200_TILE_MANY_F64 103121
#endif
#ifndef TREESAP_B200_TILE_MANY_F32
#define TREESAP_B200_TILE_MANY_F32 107121
#endif
#ifndef TREESAP_B200_QUEUE_MAX_COMPONENTS
#define TREESAP_B200_QUEUE_MAX_COMPONENTS 4
#endif
constexpr int kQueueMaxComponents = TREESAP_B200_QUEUE_MAX_COMPONENTS;
template <typename T, int G, int NC> struct DefaultTile {
    static constexpr bool kQueue = NC <= kQueueMaxComponents;
    using Spec = std::conditional_t<
        kQueue,
        std::conditional_t<sizeof(T) == 8, TileSpec<TREESAP_B200_TILE_F64>, TileSpec<TREESAP_B200_TILE_F32>>,
        std::conditional_t<sizeof(T) == 8, TileSpec<TREESAP_B200_TILE_MANY_F64>, TileSpec<TREESAP_B200_TILE_MANY_F32>>>;
    static constexpr bool kRot = (sizeof(T) == 8 ? TREESAP_B200_QROT_F64 : TREESAP_B200_QROT_F32) != 0 && kQueue;
    template <int CX, int TY, int P, int MINB, int U, int CY = 1>
    using C = treesap_b200::TileCfg<CX, TY, G, NC, T, P, MINB, U, CY, kRot && U == 1 && CX == 1 && CY == 1, kQueue>;
    using Pref = C<Spec::CX, Spec::TY, Spec::P, Spec::MINB, Spec::U, Spec::CY>;
    using type = std::conditional_t<
        Pref::fits, Pref,
        std::conditional_t<
            C<1, 3, 2, 2, 1>::fits, C<1, 3, 2, 2, 1>,
            std::conditional_t<C<1, 3, 2, 1, 1>::fits, C<1, 3, 2, 1, 1>,
                               std::conditional_t<C<1, 2, 1, 1, 1>::fits, C<1, 2, 1, 1, 1>, C<1, 1, 1, 1, 1>>>>>;
};
} // namespace detail

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType>
class SingleLevelIntegrator : public Integrator<PDEModelType> {
  protected:
    using Base = Integrator<PDEModelType>;
    using Base::ncomp;
    using Base::ngrow;
    using typename Base::BCType;
    using typename Base::InitType;
    using typename Base::RHSType;
    using Base::model;
    using Base::steps;
    using Base::time;
    using Field = treesap_b200::DeviceField<amrex::Real>;

  public:
    /// `slab` / `slab_depth`: this integrator owns planes [slab.zoff, slab.zoff + slab_depth) of the
    /// model's domain (a z slab, see ZSlabDomain.hpp); the default is the whole domain.
    SingleLevelIntegrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr,
                          treesap_b200::SlabZ slab = {}, int slab_depth = 0)
        : Base(std::move(model_)), ctx(ctx_ ? ctx_ : treesap_b200::default_context()),
          geom(model.get_geometry().data()), slab_(slab), slab_depth_(slab_depth), state_old(extent(), ngrow, ncomp),
          state_new(extent(), ngrow, ncomp) {
        if (slab_.nz > 0 && (slab_depth_ < ngrow || slab_.zoff < 0 || slab_.zoff + slab_depth_ > slab_.nz ||
                             slab_.nz != geom.domain.length(2)))
            throw std::invalid_argument("z slab outside the domain or thinner than the ghost width");
        for (int d = 0; d < 3; ++d) {
            if (block_size[d] < 1) throw std::invalid_argument("block_size must be positive");
            if (geom.domain.length(d) < ngrow) throw std::invalid_argument("domain smaller than the ghost width");
        }
        if (geom.domain.smallEnd(0) != 0 || geom.domain.smallEnd(1) != 0 || geom.domain.smallEnd(2) != 0)
            throw std::invalid_argument("treesap-b200 expects a domain index range starting at 0");
        const auto& recs = model.get_bc_recs();
        treesap_b200::cuda_check(cudaMalloc(&bc_recs_dev, sizeof(amrex::BCRec) * (recs.size() ? recs.size() : 1)),
                                 "cudaMalloc(bc_recs)");
        if (!recs.empty())
            treesap_b200::cuda_check(cudaMemcpy(bc_recs_dev, recs.data(), sizeof(amrex::BCRec) * recs.size(),
                                                cudaMemcpyHostToDevice),
                                     "cudaMemcpy(bc_recs)");
    }

    virtual ~SingleLevelIntegrator() {
        if (finite_flag) cudaFree(finite_flag);
        if (staging) cudaFree(staging);
        if (bc_recs_dev) cudaFree(bc_recs_dev);
    }

    SingleLevelIntegrator(const SingleLevelIntegrator&) = delete;
    SingleLevelIntegrator& operator=(const SingleLevelIntegrator&) = delete;

    void configureExporter(const fs::path& path, int export_interval) {
        exporter.emplace([this](double* host) { get_state(host); }, model.get_geometry(), model.get_comp_names(), path,
                         export_interval);
    }

    void initialise_impl() override {
        const auto& L = state_old.layout();
        const long long ncell = L.valid_cells();
        long long blocks = (ncell + 255) / 256;
        if (blocks > 32LL * sm_count()) blocks = 32LL * sm_count();
        treesap_b200::init_kernel<ncomp, InitType>
            <<<int(blocks), 256, 0, stream()>>>(state_old.data(), L, geom, model.get_init(), slab_.zoff);
        treesap_b200::cuda_check(cudaGetLastError(), "init_kernel launch");
        steps = 0;
        time = 0.0;
    }

    void pre_step() final override {
        if (exporter) exporter->exportIfNecessary(int(steps), time);
        fills_this_step_ = 0;
        FillPatch(state_old, time);
    }

    amrex::Real step_impl() final override { return computeNewState(model.dt_hint()); }

    void post_step() final override { swap(state_old, state_new); }

    // ---------------------------------------------------------------- treesap-b200 extensions
    ts_context* context() const { return ctx; }
    cudaStream_t stream() const { return static_cast<cudaStream_t>(ts_context_stream(ctx)); }
    int sm_count() const { return ts_context_sm_count(ctx); }
    const Field& state() const { return state_old; }
    Field& state() { return state_old; }

    /// Copies the valid cells ([comp][z][y][x], FP64) into state_old; resets time and steps.
    void set_state(const double* src, bool src_on_device = false) {
        ensure_staging();
        const auto& L = state_old.layout();
        const size_t bytes = sizeof(double) * size_t(L.valid_cells()) * ncomp;
        treesap_b200::cuda_check(cudaMemcpyAsync(staging, src, bytes,
                                                 src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                                 stream()),
                                 "cudaMemcpyAsync(set_state)");
        treesap_b200::launch_pack(state_old.data(), L, staging, 0, sm_count(), stream());
        steps = 0;
        time = 0.0;
    }

    /// Copies the valid cells of state_old out; waits for the stream when dst is on the host.
    void get_state(double* dst, bool dst_on_device = false) {
        ensure_staging();
        const auto& L = state_old.layout();
        const size_t bytes = sizeof(double) * size_t(L.valid_cells()) * ncomp;
        treesap_b200::launch_pack(state_old.data(), L, staging, 1, sm_count(), stream());
        treesap_b200::cuda_check(cudaMemcpyAsync(dst, staging, bytes,
                                                 dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                                 stream()),
                                 "cudaMemcpyAsync(get_state)");
        if (!dst_on_device) treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
    }

    /// Health check: waits for the stream and reports whether every valid cell of the state is
    /// finite (no NaN, no infinity).
    bool state_is_finite() {
        if (!finite_flag)
            treesap_b200::cuda_check(cudaMalloc(&finite_flag, sizeof(int)), "cudaMalloc(finite flag)");
        treesap_b200::cuda_check(cudaMemsetAsync(finite_flag, 0, sizeof(int), stream()), "cudaMemsetAsync(flag)");
        treesap_b200::launch_nonfinite(state_old.data(), state_old.layout(), finite_flag, sm_count(), stream());
        int h = 0;
        treesap_b200::cuda_check(cudaMemcpyAsync(&h, finite_flag, sizeof(int), cudaMemcpyDeviceToHost, stream()),
                                 "cudaMemcpyAsync(flag)");
        treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
        return h == 0;
    }

    /// Attach (or detach with nullptr) a per-launch device clock.
    void attach_clock(KernelClock* c) { clock_ = c; }

    /// Launch-shape overrides for the fused stage kernels (0 = automatic): tile rows
    /// (consumer warps per CTA) and the number of z chunks. Used by the autotuner.
    void set_launch_shape(int rows, int chunks) {
        tile_rows = rows;
        z_chunks = chunks;
    }

    /// Kernel launches enqueued by the last step() (for launch accounting).
    long long launches_per_step() const { return launches_per_step_; }

    /// Runs the host-side bookkeeping of one step (buffer swaps, clock) without enqueuing any
    /// device work: used when the step's kernels are replayed from a captured CUDA graph.
    void step_host_only() {
        dry_run_ = true;
        try {
            this->step();
        } catch (...) {
            dry_run_ = false;
            throw;
        }
        dry_run_ = false;
    }

  protected:
    virtual amrex::Real computeNewState(amrex::Real dt_hint) = 0;

    /// Ghost cells outside a non-periodic domain are never written by the stage kernels, so
    /// when no direction is periodic and the BC functor's values depend neither on time nor on
    /// the valid cells (BCType::is_time_independent and BCType::is_interior_independent), the
    /// ghost cells of a buffer keep the values of its first fill: later fills are skipped.
    static constexpr bool static_ghost_values =
        requires { requires BCType::is_time_independent && BCType::is_interior_independent; };
    bool ghosts_are_static() const {
        return static_ghost_values && !(geom.is_periodic[0] || geom.is_periodic[1] || geom.is_periodic[2]);
    }
    /// Whether a ghost fill of buffer `buf` must be enqueued now (records it as filled).
    bool ghost_fill_needed(const void* buf) {
        if (!ghosts_are_static()) return true;
        for (const void* p : ghosts_filled_)
            if (p == buf) return false;
        ghosts_filled_.push_back(buf);
        return true;
    }
    /// Counts an enqueued ghost fill towards launches_per_step().
    void count_fill() { ++fills_this_step_; }

    /// Ghost fill of an FP64 field with the model's BC functor (SingleLevelIntegrator.hpp:153-163).
    /// For a z slab the halo hook first copies the neighbouring slabs' boundary planes into the
    /// exchange ghost planes; the ghost fill then completes every other ghost cell.
    void FillPatch(Field& f, amrex::Real time_) {
        ScopedTimer timer("Integrator::FillPatch()");
        if (dry_run_) return;
        halo(f);
        if (!ghost_fill_needed(f.data())) return;
        count_fill();
        clock_begin(0);
        treesap_b200::launch_ghost_fill(f.data(), f.layout(), geom, model.get_bc(), bc_recs_dev, time_,
                                        treesap_b200::GhostMode::Functor, sm_count(), stream(), slab_);
        clock_end();
    }

  public:
    /// Where this integrator sits in a z-slab decomposition (zoff = global z of its plane 0).
    const treesap_b200::SlabZ& slab() const { return slab_; }
    /// A stage register of any element type: its data and layout.
    struct FieldRef {
        void* data;
        treesap_b200::Layout L;
    };
    /// Called before every ghost fill with the field whose exchange ghost planes must be filled
    /// from the neighbouring slabs (the same stage register of every slab).
    using HaloHook = std::function<void(const FieldRef&)>;
    void set_halo_hook(HaloHook hook) { halo_hook_ = std::move(hook); }

  protected:
    /// The halo exchange of field f (when this integrator is a slab with exchange faces).
    template <class T> void halo(treesap_b200::DeviceField<T>& f) {
        if (!halo_hook_ || dry_run_) return;
        halo_hook_(FieldRef{f.data(), f.layout()});
        count_fill();
    }

    /// Applies a pending injected stage fault of the context (ts_context_inject_fault,
    /// TS_FAULT_SKIP_COPY) to the launch about to be enqueued.
    template <class T> void take_stage_fault(treesap_b200::StageParams<T>& sp) {
        int plane = -1;
        unsigned long long wait_ns = 0;
        if (ts_context_take_stage_fault(ctx, &plane, &wait_ns)) {
            sp.skip_plane = plane;
            sp.wait_ns = wait_ns;
        }
    }

    const CUtensorMap& tensor_map(const void* base, const treesap_b200::Layout& L, int dtype, int box_x, int box_y) {
        return tmaps.get(base, L, dtype, box_x, box_y);
    }

    /// TMA descriptors of a stage launch's centre-operand fields (cached like tensor_map).
    template <class Launcher, class Params>
    treesap_b200::CentreMaps centre_maps(const Params& ep, const treesap_b200::LaunchShape& shape) {
        return Launcher::centre_maps(
            [this](const void* b, const treesap_b200::Layout& L, int dtype, int bx, int by) -> const CUtensorMap& {
                return tmaps.get(b, L, dtype, bx, by);
            },
            ep, shape);
    }

    static const int* extent_of(const amrex::Geometry& g, int* n) {
        for (int d = 0; d < 3; ++d) n[d] = g.Domain().length(d);
        return n;
    }
    /// Cells of this integrator's box: the domain, or the z slab.
    const int* extent() {
        extent_of(model.get_geometry(), extent_buf);
        if (slab_.nz > 0) extent_buf[2] = slab_depth_;
        return extent_buf;
    }

    void ensure_staging() {
        if (!staging)
            treesap_b200::cuda_check(
                cudaMalloc(&staging, sizeof(double) * size_t(state_old.layout().valid_cells()) * ncomp),
                "cudaMalloc(staging)");
    }

    ts_context* ctx;
    int extent_buf[3] = {0, 0, 0};
    amrex::GeometryData geom;
    treesap_b200::SlabZ slab_; // z-slab placement (default: the whole domain)
    int slab_depth_ = 0;
    HaloHook halo_hook_;
    Field state_old;
    Field state_new;
    amrex::BCRec* bc_recs_dev = nullptr;
    double* staging = nullptr;
    int* finite_flag = nullptr; // device flag of state_is_finite()
    treesap_b200::TensorMapCache tmaps;
    long long launches_per_step_ = 0;
    long long fills_this_step_ = 0;          // ghost fills enqueued by the current step
    std::vector<const void*> ghosts_filled_; // buffers whose static ghost cells are filled
    bool dry_run_ = false; // true while step_host_only() runs: no kernel launches
    KernelClock* clock_ = nullptr;
    void clock_begin(int cls) {
        if (clock_) clock_->begin(cls, stream());
    }
    void clock_end() {
        if (clock_) clock_->end(stream());
    }
    int tile_rows = 0;     // 0: chosen per launch (engine/stage_kernel.cuh choose_ty)
    int z_chunks = 0;      // 0: chosen per launch (make_shape)

  private:
    std::optional<PlotExporter> exporter = std::nullopt;
};

} // namespace treesap
