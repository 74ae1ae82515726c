// treesap-b200 (no reference counterpart): many independent single-box RK4 integrations in
// one set of launches.
//
// A batch holds N instances of one PDE model type, each with its own domain size, geometry,
// time step and functor parameters (a vector of PDEModel objects, as N separate
// SingleLevelRK4Integrator would take). One RK4 step of the whole batch is
//   * per stage ONE persistent launch of the fused stage kernel (engine/stage_kernel.cuh,
//     batch_stage_kernel) whose CTAs walk a host-built work list of (instance, tile, z range)
//     items, longest first, with the TMA descriptors, stage parameters, functors and
//     epilogue parameters of every instance in a device table;
//   * per ghost fill ONE launch over the ghost cells of all instances;
// and the step is captured into a CUDA graph per buffer parity. The per-cell arithmetic is
// the single-box integrators' (SingleLevelRK4Integrator, SingleLevelRK4F32StageIntegrator),
// so every instance's result is bitwise identical to its own single-box run.
//
// The tile height and the z-range length of the work items come from set_launch_shape or from
// autotune(), which times candidate shapes on the batch itself and keeps the fastest.
// Requirements: an autonomous right-hand side with time-independent, interior-independent
// boundary data (graph replays reuse the captured stage parameters); for the FP32-stage form
// the model must satisfy AffineRHSConcept.
#pragma once

#include <algorithm>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "../SingleLevelIntegrator.hpp"

namespace treesap {

namespace detail {
template <class RHS, bool F32> struct BatchLinear {
    using type = RHS;
};
template <class RHS> struct BatchLinear<RHS, true> {
    using type = decltype(linear_part_of(std::declval<const RHS&>()));
};
} // namespace detail

template <typename PDEModelType, bool F32Stage = false>
    requires PDEModelConcept<PDEModelType>
class BatchedRK4Integrator {
  public:
    using RHSType = typename PDEModelType::rhs_t;
    using BCType = typename PDEModelType::bc_t;
    using InitType = typename PDEModelType::init_t;
    static constexpr int ncomp = RHSType::ncomp;
    static constexpr int ngrow = RHSType::ngrow;
    using LinearRHS = typename detail::BatchLinear<RHSType, F32Stage>::type;
    using Tile64 = typename detail::DefaultTile<double, ngrow, ncomp>::type;
    using Tile32 = typename detail::DefaultTile<float, ngrow, ncomp>::type;
    using Field = treesap_b200::DeviceField<double>;
    using FieldF = treesap_b200::DeviceField<float>;

    static_assert(requires { requires BCType::is_time_independent && BCType::is_interior_independent; },
                  "batched stepping replays captured stage parameters: boundary data must be static");
    static_assert(!F32Stage || AffineRHSConcept<RHSType>, "the FP32-stage form needs an affine autonomous RHS");

    BatchedRK4Integrator(std::vector<PDEModelType> models_, ts_context* ctx_ = nullptr)
        : models(std::move(models_)), ctx(ctx_ ? ctx_ : treesap_b200::default_context()) {
        if (models.empty()) throw std::invalid_argument("empty batch");
        int dev = 0;
        treesap_b200::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        for (auto& m : models) {
            Inst in;
            in.geom = m.get_geometry().data();
            for (int d = 0; d < 3; ++d) {
                if (in.geom.domain.smallEnd(d) != 0)
                    throw std::invalid_argument("treesap-b200 expects a domain index range starting at 0");
                in.n[d] = in.geom.domain.length(d);
                if (in.n[d] < ngrow) throw std::invalid_argument("domain smaller than the ghost width");
            }
            in.dt = m.dt_hint();
            in.u[0] = Field(in.n, ngrow, ncomp);
            in.u[1] = Field(in.n, ngrow, ncomp);
            in.a = Field(in.n, ngrow, ncomp);
            if constexpr (F32Stage) {
                in.d1 = FieldF(in.n, ngrow, ncomp);
                in.d2 = FieldF(in.n, ngrow, ncomp);
                lins.push_back(linear_part_of(m.get_rhs()));
            } else {
                in.b = Field(in.n, ngrow, ncomp);
                lins.push_back(m.get_rhs());
            }
            insts.push_back(std::move(in));
        }
        treesap_b200::cuda_check(cudaEventCreate(&ev0), "cudaEventCreate");
        treesap_b200::cuda_check(cudaEventCreate(&ev1), "cudaEventCreate");
    }

    ~BatchedRK4Integrator() {
        drop_graphs();
        free_plans();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (staging) cudaFree(staging);
    }

    BatchedRK4Integrator(const BatchedRK4Integrator&) = delete;
    BatchedRK4Integrator& operator=(const BatchedRK4Integrator&) = delete;

    int size() const { return int(insts.size()); }
    ts_context* context() const { return ctx; }
    cudaStream_t stream() const { return static_cast<cudaStream_t>(ts_context_stream(ctx)); }
    long long steps() const { return nsteps_done; }
    double time(int i) const { return insts.at(i).time; }

    /// initialise() of every instance (Integrator.hpp:75-78): the model's InitConcept at cell centres.
    void initialise() {
        for (int i = 0; i < size(); ++i) initialise(i);
    }
    /// initialise() of instance i only (its time restarts at 0).
    void initialise(int i) {
        auto& in = insts.at(i);
        const auto& L = in.u[cur()].layout();
        long long blocks = (L.valid_cells() + 255) / 256;
        if (blocks > 4096) blocks = 4096;
        treesap_b200::init_kernel<ncomp, InitType>
            <<<int(blocks), 256, 0, stream()>>>(in.u[cur()].data(), L, in.geom, models[i].get_init());
        treesap_b200::cuda_check(cudaGetLastError(), "init_kernel launch");
        in.time = 0.0;
    }

    /// Valid cells of instance i ([comp][z][y][x], FP64) in / out (host or device pointers).
    void set_state(int i, const double* src, bool on_device = false) {
        auto& in = insts.at(i);
        ensure_staging();
        const auto& L = in.u[cur()].layout();
        treesap_b200::cuda_check(cudaMemcpyAsync(staging, src, sizeof(double) * size_t(L.valid_cells()) * ncomp,
                                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                                 stream()),
                                 "cudaMemcpyAsync(set_state)");
        treesap_b200::launch_pack(in.u[cur()].data(), L, staging, 0, sm_count(), stream());
        in.time = 0.0;
    }
    void get_state(int i, double* dst, bool on_device = false) {
        auto& in = insts.at(i);
        ensure_staging();
        const auto& L = in.u[cur()].layout();
        treesap_b200::launch_pack(in.u[cur()].data(), L, staging, 1, sm_count(), stream());
        treesap_b200::cuda_check(cudaMemcpyAsync(dst, staging, sizeof(double) * size_t(L.valid_cells()) * ncomp,
                                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                                 stream()),
                                 "cudaMemcpyAsync(get_state)");
        if (!on_device) treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
    }

    /// Tile rows and z-range length of the work items (0 = automatic); invalidates the plans.
    void set_launch_shape(int rows, int zchunk) {
        rows_ = rows;
        rows32_ = 0;
        zchunk_ = zchunk;
        drop_graphs();
        free_plans();
    }
    /// Tile rows of the FP32-input stages of the FP32-stage form (0 = those of set_launch_shape).
    void set_fp32_rows(int rows) {
        rows32_ = rows;
        drop_graphs();
        free_plans();
    }
    std::pair<int, int> launch_shape() const { return {rows_, zchunk_}; }

    /// Capture each buffer parity's step into a CUDA graph and replay it (enable), or launch
    /// kernel by kernel.
    void use_graph(bool enable) {
        graphs_on = enable;
        if (!enable) drop_graphs();
    }

    /// Advances every instance by nsteps RK4 steps (asynchronous; see last_step_timing).
    void step(int nsteps) {
        ensure_plans();
        cudaStream_t s = stream();
        treesap_b200::cuda_check(cudaEventRecord(ev0, s), "cudaEventRecord");
        long long launches = 0;
        for (int q = 0; q < nsteps; ++q) {
            const int p = cur();
            const bool with_fills = fills_needed(p);
            // static ghost cells: graphs without fills once both parities' buffers are filled
            if (graphs_on && (!ghosts_static() || fills_done[p])) {
                if (!graph[p]) {
                    cudaGraph_t g;
                    treesap_b200::cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal),
                                             "cudaStreamBeginCapture");
                    long long n = 0;
                    try {
                        n = enqueue_step(p, with_fills);
                    } catch (...) {
                        cudaStreamEndCapture(s, &g);
                        throw;
                    }
                    treesap_b200::cuda_check(cudaStreamEndCapture(s, &g), "cudaStreamEndCapture");
                    treesap_b200::cuda_check(cudaGraphInstantiate(&graph[p], g, 0), "cudaGraphInstantiate");
                    cudaGraphDestroy(g);
                    graph_launches[p] = n;
                }
                treesap_b200::cuda_check(cudaGraphLaunch(graph[p], s), "cudaGraphLaunch");
                launches += graph_launches[p];
            } else {
                launches += enqueue_step(p, with_fills);
            }
            fills_done[p] = true;
            for (auto& in : insts) in.time += in.dt;
            ++nsteps_done;
        }
        treesap_b200::cuda_check(cudaEventRecord(ev1, s), "cudaEventRecord");
        last_launches = launches;
    }

    /// Device time (ms, after the stream completed) and kernel launches of the last step() call.
    std::pair<double, long long> last_step_timing() const {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        return {double(ms), last_launches};
    }

    /// Times candidate launch shapes (tile rows x z-range lengths) on this batch, trial_steps
    /// steps each after one warm-up step, keeps the fastest and returns it. The instances'
    /// states are saved before and restored after the trials.
    std::pair<int, int> autotune(int trial_steps = 3) {
        const int tymax = Tile64::TYMAX < Tile32::TYMAX ? Tile64::TYMAX : Tile32::TYMAX;
        std::vector<Field> saved;
        std::vector<double> saved_t;
        for (auto& in : insts) {
            saved.emplace_back(in.n, ngrow, ncomp);
            treesap_b200::cuda_check(cudaMemcpyAsync(saved.back().data(), in.u[cur()].data(),
                                                     size_t(in.u[cur()].layout().bytes()), cudaMemcpyDeviceToDevice,
                                                     stream()),
                                     "cudaMemcpyAsync(save)");
            saved_t.push_back(in.time);
        }
        const long long saved_steps = nsteps_done;
        const bool saved_graphs = graphs_on;
        graphs_on = false;
        double best = 1e300;
        std::pair<int, int> best_shape{0, 0};
        const int zchunks[] = {0, 64, 32, 16};
        for (int ty = tymax; ty >= 2; --ty) {
            for (int zc : zchunks) {
                if (zc != 0 && zc < 4 * ngrow) continue;
                set_launch_shape(ty, zc);
                step(1);
                step(trial_steps);
                treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
                const double ms = last_step_timing().first;
                if (ms < best) {
                    best = ms;
                    best_shape = {ty, zc};
                }
            }
        }
        set_launch_shape(best_shape.first, best_shape.second);
        if constexpr (F32Stage) {
            // the FP32-input stages (two cells per thread) may prefer other tile rows than the
            // FP64-input ones: refine them with the FP64 rows and z ranges fixed
            int best32 = 0;
            for (int ty = Tile32::TYMAX; ty >= 2; --ty) {
                if (ty == best_shape.first) continue;
                set_fp32_rows(ty);
                step(1);
                step(trial_steps);
                treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
                const double ms = last_step_timing().first;
                if (ms < best) {
                    best = ms;
                    best32 = ty;
                }
            }
            set_fp32_rows(best32);
            // and the FP64-input stages with those FP32 rows
            const int r32 = best32 > 0 ? best32 : best_shape.first;
            int best64 = best_shape.first;
            for (int ty = Tile64::TYMAX; ty >= 2; --ty) {
                if (ty == best_shape.first) continue;
                set_launch_shape(ty, best_shape.second);
                set_fp32_rows(r32);
                step(1);
                step(trial_steps);
                treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
                const double ms = last_step_timing().first;
                if (ms < best) {
                    best = ms;
                    best64 = ty;
                }
            }
            best_shape.first = best64;
            set_launch_shape(best64, best_shape.second);
            set_fp32_rows(r32);
        }
        // restore the states into the saved parity's buffers, ghost cells included
        nsteps_done = saved_steps;
        fills_done[0] = fills_done[1] = false;
        for (int i = 0; i < size(); ++i) {
            auto& in = insts[i];
            treesap_b200::cuda_check(cudaMemcpyAsync(in.u[cur()].data(), saved[i].data(),
                                                     size_t(in.u[cur()].layout().bytes()), cudaMemcpyDeviceToDevice,
                                                     stream()),
                                     "cudaMemcpyAsync(restore)");
            in.time = saved_t[i];
        }
        treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
        graphs_on = saved_graphs;
        return best_shape;
    }

    /// Work items per stage launch of the FP64 / FP32 tile configurations (after a step).
    std::pair<int, int> items_per_launch() const { return {items64.n, items32.n}; }

  private:
    using RG = treesap_b200::GhostEntry<double, BCType>;
    using RGF = treesap_b200::GhostEntry<float, BCType>;

    struct Inst {
        int n[3] = {0, 0, 0};
        amrex::GeometryData geom{};
        double dt = 0.0, time = 0.0;
        Field u[2];   // state, swapped every step
        Field a, b;   // FP64 form: the two stage arguments; FP32-stage form: a = k0
        FieldF d1, d2; // FP32-stage form: stage differences
    };

    template <class T> struct DevArray {
        T* p = nullptr;
        int n = 0;
        void upload(const T* h, int count, cudaStream_t s) {
            release();
            n = count;
            if (!n) return;
            treesap_b200::cuda_check(cudaMalloc(&p, sizeof(T) * size_t(n)), "cudaMalloc(batch table)");
            treesap_b200::cuda_check(cudaMemcpyAsync(p, h, sizeof(T) * size_t(n), cudaMemcpyHostToDevice, s),
                                     "cudaMemcpyAsync(batch table)");
            // the host table may go away after this call
            treesap_b200::cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        }
        void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), int(h.size()), s); }
        void release() {
            if (p) cudaFree(p);
            p = nullptr;
            n = 0;
        }
    };

    template <class Cfg, class R, class Epi> struct StagePlan {
        using Entry = treesap_b200::StageEntry<Cfg, R, Epi>;
        DevArray<Entry> entries;
        static auto kernel() { return &treesap_b200::batch_stage_kernel<Cfg, R, Epi>; }
        /// Persistent grid for tiles of `ty` rows: the CTAs of 32 ty + 32 threads that fit an SM
        /// at once (registers and the ring's shared memory), times the SMs.
        static int grid(int sms, int ty) {
            using RingT = treesap_b200::Ring<Cfg, Epi>;
            return treesap_b200::cached_occupancy<&treesap_b200::batch_stage_kernel<Cfg, R, Epi>, Cfg::TYMAX>(
                       ty, RingT::SMEM) *
                   sms;
        }
        void launch(const DevArray<treesap_b200::ItemBox>& items, int ty, int* err, int sms, cudaStream_t s) const {
            using RingT = treesap_b200::Ring<Cfg, Epi>;
            int g = grid(sms, ty);
            if (g > items.n) g = items.n;
            if (g < 1) return;
            // through the registered entry point, like StageLauncher::launch
            const Entry* e = entries.p;
            const treesap_b200::ItemBox* it = items.p;
            int n = int(items.n);
            void* args[] = {&e, &it, &n, &ty, &err};
            treesap_b200::cuda_check(cudaLaunchKernel(reinterpret_cast<const void*>(kernel()), dim3(g),
                                                      dim3(32 * ty + 32), args, size_t(RingT::SMEM), s),
                                     "batch_stage_kernel launch");
        }
    };

    template <class T> struct FillPlan {
        DevArray<treesap_b200::GhostEntry<T, BCType>> entries;
        DevArray<treesap_b200::GhostChunk> chunks;
        void launch(const amrex::BCRec* bcr, int sms, cudaStream_t s) const {
            if (chunks.n == 0) return;
            int blocks = chunks.n;
            if (blocks > 32 * sms) blocks = 32 * sms;
            treesap_b200::batch_ghost_fill_kernel<T, BCType><<<blocks, treesap_b200::kGhostFillThreads, 0, s>>>(entries.p, chunks.p, chunks.n, bcr);
            treesap_b200::cuda_check(cudaGetLastError(), "batch_ghost_fill_kernel launch");
        }
    };

    // stage plans per buffer parity
    template <int S> using EpiR = treesap_b200::EpiRK4<S>;
    struct PlanF64 {
        StagePlan<Tile64, RHSType, EpiR<0>> s0;
        StagePlan<Tile64, RHSType, EpiR<1>> s1;
        StagePlan<Tile64, RHSType, EpiR<2>> s2;
        StagePlan<Tile64, RHSType, EpiR<3>> s3;
        FillPlan<double> fill[4]; // before stages 0..3
    };
    struct PlanF32 {
        StagePlan<Tile64, RHSType, treesap_b200::EpiF32S0> s0;
        StagePlan<Tile64, LinearRHS, treesap_b200::EpiF32S1> s1;
        StagePlan<Tile32, LinearRHS, treesap_b200::EpiF32Lin<2>> s2;
        StagePlan<Tile32, LinearRHS, treesap_b200::EpiF32Lin<3>> s3;
        FillPlan<double> fill_u, fill_k0;
        FillPlan<float> fill_d1, fill_d2;
    };
    using Plan = std::conditional_t<F32Stage, PlanF32, PlanF64>;

    int cur() const { return int(nsteps_done & 1); }
    int sm_count() const { return ts_context_sm_count(ctx); }
    int* err() const { return ts_context_error_word(ctx); }

    bool ghosts_static() const {
        for (const auto& in : insts)
            if (in.geom.is_periodic[0] || in.geom.is_periodic[1] || in.geom.is_periodic[2]) return false;
        return true;
    }
    bool fills_needed(int p) const { return !(ghosts_static() && fills_done[p]); }

    void ensure_staging() {
        if (staging) return;
        size_t mx = 0;
        for (const auto& in : insts) mx = std::max(mx, size_t(in.u[0].layout().valid_cells()) * ncomp);
        treesap_b200::cuda_check(cudaMalloc(&staging, sizeof(double) * mx), "cudaMalloc(staging)");
    }

    template <class Cfg> int rows_for() const {
        if constexpr (std::is_same_v<Cfg, Tile32> && !std::is_same_v<Tile32, Tile64>)
            if (rows32_ > 0 && rows32_ <= Cfg::TYMAX) return rows32_;
        if (rows_ > 0 && rows_ <= Cfg::TYMAX) return rows_;
        return Cfg::TYMAX;
    }

    /// Work list of one tile configuration: every instance's tiles x z ranges, longest first.
    template <class Cfg> std::vector<treesap_b200::ItemBox> make_items(int ty) const {
        std::vector<treesap_b200::ItemBox> v;
        for (int i = 0; i < size(); ++i) {
            const auto& in = insts[i];
            int zc = zchunk_ > 0 ? zchunk_ : in.n[2];
            for (int z0 = 0; z0 < in.n[2]; z0 += zc)
                for (int y0 = 0; y0 < in.n[1]; y0 += ty * Cfg::CY)
                    for (int x0 = 0; x0 < in.n[0]; x0 += Cfg::TX)
                        v.push_back({i, x0, y0, z0, std::min(in.n[2], z0 + zc)});
        }
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.z1 - a.z0 > b.z1 - b.z0; });
        return v;
    }

    template <class Cfg, class Plan_, class R, class Epi, class MakeEp>
    void build_stage(Plan_& plan, const std::vector<R>& rhs, int ty, int dtype, MakeEp&& make) {
        using Entry = treesap_b200::StageEntry<Cfg, R, Epi>;
        // the functors need not be default-constructible: entries are built in raw storage
        struct Buf {
            Entry* p;
            explicit Buf(size_t n)
                : p(static_cast<Entry*>(::operator new[](sizeof(Entry) * n, std::align_val_t(alignof(Entry))))) {
                std::memset(static_cast<void*>(p), 0, sizeof(Entry) * n);
            }
            ~Buf() { ::operator delete[](p, std::align_val_t(alignof(Entry))); }
        } h(insts.size());
        for (int i = 0; i < size(); ++i) {
            auto& in = insts[i];
            const void* input = nullptr;
            treesap_b200::Layout L;
            typename Epi::Params ep = make(i, input, L);
            Entry& e = h.p[i];
            const ts_field_layout cl = L.to_c(dtype);
            treesap_b200::ts_check(ts_field_tensor_map(&cl, input, Cfg::BX, ty * Cfg::CY + 2 * Cfg::G, &e.tmap), ctx,
                                   "ts_field_tensor_map");
            for (int k = 0; k < Epi::kCentre; ++k) {
                const treesap_b200::CentreSrc c = Epi::centre_src(ep, k);
                const ts_field_layout cc = c.L.to_c(c.dtype);
                treesap_b200::ts_check(ts_field_tensor_map(&cc, c.base, Cfg::TX, ty * Cfg::CY, &e.cmaps.map[k]), ctx,
                                       "ts_field_tensor_map");
                e.cmaps.x[k] = c.L.xoff;
                e.cmaps.y[k] = c.L.g;
                e.cmaps.z[k] = c.L.g;
            }
            e.sp = treesap_b200::StageParams<typename Cfg::T>{}; // the entry's storage is raw memory
            e.sp.in = static_cast<const typename Cfg::T*>(input);
            e.sp.L = L;
            e.sp.geom = in.geom;
            e.sp.time = in.time;
            e.sp.ty = ty;
            e.sp.err = err();
            new (&e.rhs) R(rhs[i]);
            std::memcpy(static_cast<void*>(&e.ep), &ep, sizeof(ep));
        }
        plan.entries.upload(h.p, size(), stream());
    }

    template <class T> void build_fill(FillPlan<T>& f, std::vector<std::pair<T*, treesap_b200::Layout>> fields,
                                       treesap_b200::GhostMode mode) {
        std::vector<treesap_b200::GhostEntry<T, BCType>> h;
        std::vector<treesap_b200::GhostChunk> ch;
        for (int i = 0; i < size(); ++i) {
            h.push_back(treesap_b200::GhostEntry<T, BCType>{fields[i].first, fields[i].second, insts[i].geom,
                                                            models[i].get_bc(), insts[i].time, int(mode)});
            const long long total = treesap_b200::ghost_count(fields[i].second).total();
            for (long long c = 0; c < total; c += treesap_b200::kGhostChunk) ch.push_back({i, 0, c});
        }
        f.entries.upload(h, stream());
        f.chunks.upload(ch, stream());
    }

    void ensure_plans() {
        if (plans_ready) return;
        using namespace treesap_b200;
        const int ty64 = rows_for<Tile64>(), ty32 = rows_for<Tile32>();
        ty_[0] = ty64;
        ty_[1] = ty32;
        const auto i64 = make_items<Tile64>(ty64);
        items64.upload(i64, stream());
        const auto i32 = make_items<Tile32>(ty32);
        items32.upload(i32, stream());
        std::vector<RHSType> rhs;
        for (int i = 0; i < size(); ++i) rhs.push_back(models[i].get_rhs());
        const std::vector<LinearRHS>& lin = lins;
        constexpr double af[4] = {0.0, 0.5, 0.5, 1.0};
        constexpr double bf[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
        for (int p = 0; p < 2; ++p) {
            Plan& P = plan[p];
            auto oldf = [&](int i) -> Field& { return insts[i].u[p]; };
            auto newf = [&](int i) -> Field& { return insts[i].u[1 - p]; };
            if constexpr (!F32Stage) {
                // stage arguments: this parity starts with (arg, arg_next) = (X, Y)
                auto X = [&](int i) -> Field& { return p == 0 ? insts[i].a : insts[i].b; };
                auto Y = [&](int i) -> Field& { return p == 0 ? insts[i].b : insts[i].a; };
                build_stage<Tile64, decltype(P.s0), RHSType, EpiRK4<0>>(
                    P.s0, rhs, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = oldf(i).data();
                        L = oldf(i).layout();
                        const double dt = insts[i].dt;
                        return EpiRK4<0>::Params{newf(i).data(), Y(i).data(), oldf(i).data(), L, dt * bf[0],
                                                 dt * af[1]};
                    });
                build_stage<Tile64, decltype(P.s1), RHSType, EpiRK4<1>>(
                    P.s1, rhs, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = Y(i).data();
                        L = Y(i).layout();
                        const double dt = insts[i].dt;
                        return EpiRK4<1>::Params{newf(i).data(), X(i).data(), oldf(i).data(), L, dt * bf[1],
                                                 dt * af[2]};
                    });
                build_stage<Tile64, decltype(P.s2), RHSType, EpiRK4<2>>(
                    P.s2, rhs, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = X(i).data();
                        L = X(i).layout();
                        const double dt = insts[i].dt;
                        return EpiRK4<2>::Params{newf(i).data(), Y(i).data(), oldf(i).data(), L, dt * bf[2],
                                                 dt * af[3]};
                    });
                build_stage<Tile64, decltype(P.s3), RHSType, EpiRK4<3>>(
                    P.s3, rhs, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = Y(i).data();
                        L = Y(i).layout();
                        const double dt = insts[i].dt;
                        return EpiRK4<3>::Params{newf(i).data(), X(i).data(), oldf(i).data(), L, dt * bf[3], 0.0};
                    });
                auto fields = [&](auto&& which) {
                    std::vector<std::pair<double*, Layout>> v;
                    for (int i = 0; i < size(); ++i) v.push_back({which(i).data(), which(i).layout()});
                    return v;
                };
                build_fill(P.fill[0], fields(oldf), GhostMode::Functor);
                build_fill(P.fill[1], fields(Y), GhostMode::Functor);
                build_fill(P.fill[2], fields(X), GhostMode::Functor);
                build_fill(P.fill[3], fields(Y), GhostMode::Functor);
            } else {
                build_stage<Tile64, decltype(P.s0), RHSType, EpiF32S0>(
                    P.s0, rhs, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = oldf(i).data();
                        L = oldf(i).layout();
                        return EpiF32S0::Params{insts[i].a.data(), newf(i).data(), L, insts[i].dt};
                    });
                build_stage<Tile64, decltype(P.s1), LinearRHS, EpiF32S1>(
                    P.s1, lin, ty64, TS_F64, [&](int i, const void*& in, Layout& L) {
                        in = insts[i].a.data();
                        L = insts[i].a.layout();
                        return EpiF32S1::Params{insts[i].d1.data(), insts[i].d1.layout(), 0.5 * insts[i].dt};
                    });
                auto lin_ep = [&](int i, int S) {
                    EpiF32Lin<2>::Params ep{};
                    ep.d_out = S < 3 ? insts[i].d2.data() : nullptr;
                    ep.d1 = insts[i].d1.data();
                    ep.u = newf(i).data();
                    ep.Lf = insts[i].d1.layout();
                    ep.Lu = newf(i).layout();
                    ep.a_dt = float(S < 3 ? 0.5 * insts[i].dt : insts[i].dt);
                    ep.dt = insts[i].dt;
                    return ep;
                };
                build_stage<Tile32, decltype(P.s2), LinearRHS, EpiF32Lin<2>>(
                    P.s2, lin, ty32, TS_F32, [&](int i, const void*& in, Layout& L) {
                        in = insts[i].d1.data();
                        L = insts[i].d1.layout();
                        return lin_ep(i, 2);
                    });
                build_stage<Tile32, decltype(P.s3), LinearRHS, EpiF32Lin<3>>(
                    P.s3, lin, ty32, TS_F32, [&](int i, const void*& in, Layout& L) {
                        in = insts[i].d2.data();
                        L = insts[i].d2.layout();
                        const auto e2 = lin_ep(i, 3);
                        EpiF32Lin<3>::Params ep{};
                        ep.d_out = e2.d_out;
                        ep.d1 = e2.d1;
                        ep.u = e2.u;
                        ep.Lf = e2.Lf;
                        ep.Lu = e2.Lu;
                        ep.a_dt = e2.a_dt;
                        ep.dt = e2.dt;
                        return ep;
                    });
                std::vector<std::pair<double*, Layout>> fu, fk;
                std::vector<std::pair<float*, Layout>> f1, f2;
                for (int i = 0; i < size(); ++i) {
                    fu.push_back({oldf(i).data(), oldf(i).layout()});
                    fk.push_back({insts[i].a.data(), insts[i].a.layout()});
                    f1.push_back({insts[i].d1.data(), insts[i].d1.layout()});
                    f2.push_back({insts[i].d2.data(), insts[i].d2.layout()});
                }
                build_fill(P.fill_u, fu, GhostMode::Functor);
                build_fill(P.fill_k0, fk, GhostMode::Homogeneous);
                build_fill(P.fill_d1, f1, GhostMode::Homogeneous);
                build_fill(P.fill_d2, f2, GhostMode::Homogeneous);
            }
        }
        treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize");
        plans_ready = true;
    }

    void free_plans() {
        plans_ready = false;
        items64.release();
        items32.release();
        for (auto& P : plan) {
            P.s0.entries.release();
            P.s1.entries.release();
            P.s2.entries.release();
            P.s3.entries.release();
            if constexpr (F32Stage) {
                for (auto* f : {&P.fill_u, &P.fill_k0}) {
                    f->entries.release();
                    f->chunks.release();
                }
                for (auto* f : {&P.fill_d1, &P.fill_d2}) {
                    f->entries.release();
                    f->chunks.release();
                }
            } else {
                for (auto& f : P.fill) {
                    f.entries.release();
                    f.chunks.release();
                }
            }
        }
    }

    void drop_graphs() {
        for (auto& g : graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    /// Enqueues one step of parity p; returns the number of kernels launched.
    long long enqueue_step(int p, bool with_fills) {
        const Plan& P = plan[p];
        cudaStream_t s = stream();
        const int sms = sm_count();
        long long n = 4;
        if constexpr (!F32Stage) {
            if (with_fills) P.fill[0].launch(nullptr, sms, s);
            P.s0.launch(items64, ty_[0], err(), sms, s);
            if (with_fills) P.fill[1].launch(nullptr, sms, s);
            P.s1.launch(items64, ty_[0], err(), sms, s);
            if (with_fills) P.fill[2].launch(nullptr, sms, s);
            P.s2.launch(items64, ty_[0], err(), sms, s);
            if (with_fills) P.fill[3].launch(nullptr, sms, s);
            P.s3.launch(items64, ty_[0], err(), sms, s);
        } else {
            if (with_fills) P.fill_u.launch(nullptr, sms, s);
            P.s0.launch(items64, ty_[0], err(), sms, s);
            if (with_fills) P.fill_k0.launch(nullptr, sms, s);
            P.s1.launch(items64, ty_[0], err(), sms, s);
            if (with_fills) P.fill_d1.launch(nullptr, sms, s);
            P.s2.launch(items32, ty_[1], err(), sms, s);
            if (with_fills) P.fill_d2.launch(nullptr, sms, s);
            P.s3.launch(items32, ty_[1], err(), sms, s);
        }
        if (with_fills) n += 4;
        return n;
    }

    std::vector<PDEModelType> models;
    ts_context* ctx;
    std::vector<Inst> insts;
    std::vector<LinearRHS> lins; // per instance: the RHS (FP64 form) or its linear part (FP32-stage form)
    Plan plan[2];
    DevArray<treesap_b200::ItemBox> items64, items32;
    int ty_[2] = {0, 0};
    int rows_ = 0, rows32_ = 0, zchunk_ = 0;
    bool plans_ready = false;
    bool graphs_on = false;
    bool fills_done[2] = {false, false};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    long long graph_launches[2] = {0, 0};
    long long nsteps_done = 0;
    long long last_launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double* staging = nullptr;
};

} // namespace treesap
