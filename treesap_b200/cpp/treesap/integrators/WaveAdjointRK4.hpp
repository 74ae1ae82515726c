// treesap-b200 (no reference counterpart): discrete adjoint of RK4 for the variable-speed
// scalar wave model (rhs/WaveAdjointRHS.hpp), with checkpoint-and-recompute, and its
// tangent-linear model.
//
// Forward: u_{n+1} = RK4_L(u_n) with u = {phi, pi, c2} on a periodic grid. Loss
//   J = 1/2 sum_cells (phi_N - phi_target)^2.
// Reverse sweep: lambda_N = dJ/du_N = {phi_N - phi_target, 0}; lambda_n = RK4_{L^T}(lambda_{n+1}),
// which is the transpose of the forward step (module header of WaveAdjointRHS.hpp). The
// speed gradient follows from reverse-mode differentiation of the stage form
//   k_s = L w_s,  w_0 = u,  w_1 = u + dt/2 k_0,  w_2 = u + dt/2 k_1,  w_3 = u + dt k_2:
// the cotangent of k_{3-s} equals b_s a_s, where a_s is the argument of stage s of RK4_{L^T}
// and b = dt {1/6, 1/3, 1/3, 1/6}, so
//   dJ/dc2 = sum_n sum_s b_s  a_{s,pi}(n) * (D w_{3-s,phi})(n),     dJ/dc = 2 c dJ/dc2.
// The forward states are saved every `checkpoint_every` steps; the reverse sweep recomputes
// one segment of states from its checkpoint, then per step the forward stage arguments w_s,
// the adjoint step and four gradient launches (the Laplacian of w_{3-s} times the centre
// value a_{s,pi}). All of it runs on the fused stage kernels (engine/stage_kernel.cuh) in FP64.
#pragma once

#include <cmath>
#include <vector>

#include "../SingleLevelIntegrator.hpp"
#include "../pde-model/bcs/NoOpBC.hpp"
#include "WaveAdjointRHS.hpp"

namespace treesap_b200 {

/// g(., 0) += b * a(., 1) * k(., 0): the speed-gradient accumulation (centre operands: the
/// adjoint stage argument a (C0) and the gradient field g (C1), both 3-component FP64).
struct EpiSpeedGradient {
    struct Params {
        double* g;
        const double* a;
        Layout L;
        double b;
    };
    static constexpr int kCentre = 2;
    using C0 = double;
    using C1 = double;
    static CentreSrc centre_src(const Params& p, int k) {
        return k == 0 ? CentreSrc{p.a, p.L, TS_F64} : CentreSrc{p.g, p.L, TS_F64};
    }
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T*, int, int i0, int j, int z, const CO& co) {
        double a[CX], g[CX], out[CX];
        lds<CX>(co.c0 + 1 * co.cps, a);
        lds<CX>(co.c1, g);
#pragma unroll
        for (int e = 0; e < CX; ++e) out[e] = g[e] + p.b * a[e] * k[e][0];
        stcs<CX>(p.g + p.L.index(i0, j, z, 0), out, act);
    }
};

/// The FP32-stage form of the speed-gradient accumulation, term Q of one step:
///   g += coef_Q * D X_Q,   X_Q = u, k0 (FP64 stencils), d1, d2 (FP32 stencils),
/// where u, k0, d1, d2 are the forward step's FP32-stage registers and the forward stage
/// arguments are w0 = u, w1 = u + dt/2 k0, w2 = u + dt/2 (k0 + d1), w3 = u + dt (k0 + d2).
/// With A_s the pi component of the adjoint stage argument s (from the adjoint step's
/// registers lam, kb0, db1, db2: A0 = lam, A1 = lam + dt/2 kb0, A2 = lam + dt/2 (kb0 + db1),
/// A3 = lam + dt (kb0 + db2)) and beta_s = dt b_s, the step's term sum_s beta_s A_s D w_{3-s}
/// regroups into
///   coef_u = sum_s beta_s A_s,  coef_k0 = dt (beta_0 A0 + beta_1 A1 / 2 + beta_2 A2 / 2),
///   coef_d1 = dt / 2 beta_1 A1, coef_d2 = dt beta_0 A0.
/// The adjoint registers and g are read at the cell from global memory.
struct SpeedGradF32Params {
    double* g;
    Layout Lg;
    const double* lam;
    const double* kb0;
    Layout Lu;
    const float* db1;
    const float* db2;
    Layout Lf;
    double dt;
};
template <int Q> struct EpiSpeedGradF32 : NoCentre {
    using Params = SpeedGradF32Params;
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T*, int, int i0, int j, int z, const CO&) {
#pragma unroll
        for (int e = 0; e < CX; ++e) {
            if (!act[e]) continue;
            const long long ou = p.Lu.index(i0 + e, j, z, 1);
            const long long of = p.Lf.index(i0 + e, j, z, 1);
            const double lam = p.lam[ou], kb = p.kb0[ou];
            const double dt = p.dt, b0 = dt / 6.0, b1 = dt / 3.0;
            double coef;
            if constexpr (Q == 0) {
                const double a1 = lam + 0.5 * dt * kb, a2 = lam + 0.5 * dt * (kb + double(p.db1[of]));
                const double a3 = lam + dt * (kb + double(p.db2[of]));
                coef = b0 * lam + b1 * a1 + b1 * a2 + b0 * a3;
            } else if constexpr (Q == 1) {
                const double a1 = lam + 0.5 * dt * kb, a2 = lam + 0.5 * dt * (kb + double(p.db1[of]));
                coef = dt * (b0 * lam + 0.5 * b1 * a1 + 0.5 * b1 * a2);
            } else if constexpr (Q == 2) {
                coef = 0.5 * dt * b1 * (lam + 0.5 * dt * kb);
            } else {
                coef = dt * b0 * lam;
            }
            double* g = p.g + p.Lg.index(i0 + e, j, z, 0);
            *g += coef * double(k[e][0]);
        }
    }
};

} // namespace treesap_b200

namespace treesap {

/// Launches the four FP32-stage speed-gradient terms of one step (EpiSpeedGradF32) on the
/// registers of a forward and an adjoint FP32-stage RK4 step of the two-component wave system.
template <int G> class WaveSpeedGradientF32 {
  public:
    using Lap = tsb::WaveLaplacianRHS<G>;
    using Tile64 = typename detail::DefaultTile<double, G, 2>::type;
    using Tile32 = typename detail::DefaultTile<float, G, 2>::type;
    struct Reg {
        void* data;
        treesap_b200::Layout L;
    };

    WaveSpeedGradientF32(ts_context* ctx_, const amrex::GeometryData& geom_) : ctx(ctx_), geom(geom_) {}

    /// g += the step's speed-gradient term (g: one FP64 component, any layout of the domain).
    /// fwd, adj: the registers u, k0, d1, d2 of the forward and of the adjoint step.
    void accumulate(const Reg (&fwd)[4], const Reg (&adj)[4], double* g, const treesap_b200::Layout& Lg, double dt) {
        using namespace treesap_b200;
        const auto make = [&]() {
            SpeedGradF32Params p{};
            p.g = g;
            p.Lg = Lg;
            p.lam = static_cast<const double*>(adj[0].data);
            p.kb0 = static_cast<const double*>(adj[1].data);
            p.Lu = adj[0].L;
            p.db1 = static_cast<const float*>(adj[2].data);
            p.db2 = static_cast<const float*>(adj[3].data);
            p.Lf = adj[2].L;
            p.dt = dt;
            return p;
        };
        const auto p = make();
        term<0, double, Tile64>(fwd[0], p);
        term<1, double, Tile64>(fwd[1], p);
        term<2, float, Tile32>(fwd[2], p);
        term<3, float, Tile32>(fwd[3], p);
    }

  private:
    template <int Q, class T, class Cfg> void term(const Reg& in, const treesap_b200::SpeedGradF32Params& ep) {
        using namespace treesap_b200;
        using Epi = EpiSpeedGradF32<Q>;
        using Launcher = StageLauncher<Cfg, Lap, Epi>;
        const Layout& L = in.L;
        const int sm = ts_context_sm_count(ctx);
        const auto shape = Launcher::shape(L, sm);
        const CUtensorMap& tm = tmaps.get(in.data, L, sizeof(T) == 8 ? TS_F64 : TS_F32, Launcher::box_x(),
                                          Launcher::box_y(shape));
        const CentreMaps cm = Launcher::centre_maps(
            [this](const void* b, const Layout& Lc, int dtype, int bx, int by) -> const CUtensorMap& {
                return tmaps.get(b, Lc, dtype, bx, by);
            },
            ep, shape);
        StageParams<T> sp{};
        sp.in = static_cast<const T*>(in.data);
        sp.L = L;
        sp.geom = geom;
        sp.time = 0.0;
        sp.err = ts_context_error_word(ctx);
        Launcher::launch(tm, cm, sp, Lap{}, ep, shape, static_cast<cudaStream_t>(ts_context_stream(ctx)));
    }

    ts_context* ctx;
    amrex::GeometryData geom;
    treesap_b200::TensorMapCache tmaps;
};

template <int G> class WaveAdjointRK4 {
  public:
    static constexpr int NC = 3;   // phi, pi, c2
    static constexpr int NCT = 6;  // phi, pi, c2, dphi, dpi, dc2
    using Field = treesap_b200::DeviceField<double>;
    using Fwd = tsb::WaveC2RHS<G>;
    using Adj = tsb::WaveC2AdjointRHS<G>;
    using Lap = tsb::WaveC2LaplacianRHS<G>;
    using Tan = tsb::WaveC2TangentRHS<G>;
    using Tile = typename detail::DefaultTile<double, G, NC>::type;
    using TileT = typename detail::DefaultTile<double, G, NCT>::type;

    WaveAdjointRK4(const amrex::Geometry& geometry, double dt_, double ko_strength, int checkpoint_every_,
                   ts_context* ctx_ = nullptr)
        : ctx(ctx_ ? ctx_ : treesap_b200::default_context()), geom(geometry.data()), dt(dt_),
          every(checkpoint_every_) {
        for (int d = 0; d < 3; ++d) {
            if (!geom.is_periodic[d]) throw std::invalid_argument("the adjoint needs a periodic domain");
            if (geom.domain.smallEnd(d) != 0) throw std::invalid_argument("domain index range must start at 0");
            n[d] = geom.domain.length(d);
            if (n[d] < G) throw std::invalid_argument("domain smaller than the ghost width");
        }
        if (every < 1) throw std::invalid_argument("checkpoint interval must be >= 1");
        fwd.ko_strength = adj.ko_strength = tan.ko_strength = ko_strength;
        for (int q = 0; q < 5; ++q) work.emplace_back(n, G, NC);
        for (int q = 0; q < 5; ++q) adjf.emplace_back(n, G, NC);
        g = Field(n, G, NC);
        ncell = (long long)n[0] * n[1] * n[2];
        treesap_b200::cuda_check(cudaMalloc(&staging, sizeof(double) * size_t(ncell) * NCT), "cudaMalloc(staging)");
    }
    ~WaveAdjointRK4() {
        if (staging) cudaFree(staging);
    }
    WaveAdjointRK4(const WaveAdjointRK4&) = delete;
    WaveAdjointRK4& operator=(const WaveAdjointRK4&) = delete;

    long long cells() const { return ncell; }
    cudaStream_t stream() const { return static_cast<cudaStream_t>(ts_context_stream(ctx)); }

    /// Forward run: phi_T, pi_T (host, may be null) after nsteps from (phi0, pi0) with speed c.
    void forward(const double* phi0, const double* pi0, const double* c, int nsteps, double* phiT, double* piT) {
        upload_state(work[0], phi0, pi0, c);
        Field* a = &work[0];
        Field* b = &work[1];
        for (int s = 0; s < nsteps; ++s) {
            rk4_step(fwd, *a, *b, work[2], work[3], work[4]);
            std::swap(a, b);
        }
        download(*a, 0, phiT);
        download(*a, 1, piT);
        sync();
    }

    /// Loss and gradients: grad_phi0, grad_pi0, grad_c (host, ncell each; any may be null).
    double gradient(const double* phi0, const double* pi0, const double* c, int nsteps, const double* target,
                    double* grad_phi0, double* grad_pi0, double* grad_c) {
        const int nck = nsteps / every + 1;
        while (int(ckpt.size()) < nck) ckpt.emplace_back(n, G, NC);
        while (int(seg.size()) < every) seg.emplace_back(n, G, NC);
        // forward sweep with checkpoints
        upload_state(ckpt[0], phi0, pi0, c);
        copy(work[0], ckpt[0]);
        Field* a = &work[0];
        Field* b = &work[1];
        for (int s = 0; s < nsteps; ++s) {
            rk4_step(fwd, *a, *b, work[2], work[3], work[4]);
            std::swap(a, b);
            if ((s + 1) % every == 0 && s + 1 < nsteps) copy(ckpt[(s + 1) / every], *a);
        }
        // loss and the final adjoint lambda_N = {phi_N - target, 0, c2}
        std::vector<double> phiN(ncell), host(size_t(ncell) * NC);
        download(*a, 0, phiN.data());
        download(*a, 2, host.data() + 2 * ncell); // c2
        sync();
        double loss = 0.0;
        for (long long q = 0; q < ncell; ++q) {
            const double r = phiN[q] - target[q];
            loss += 0.5 * r * r;
            host[q] = r;
            host[ncell + q] = 0.0;
        }
        Field* lam = &adjf[0];
        Field* lamn = &adjf[1];
        upload_raw(*lam, host.data());
        treesap_b200::cuda_check(cudaMemsetAsync(g.data(), 0, size_t(g.layout().bytes()), stream()),
                                 "cudaMemsetAsync(gradient)");
        // reverse sweep, segment by segment
        for (int sg = (nsteps - 1) / every; sg >= 0; --sg) {
            const int start = sg * every, end = std::min(nsteps, start + every);
            copy(seg[0], ckpt[sg]);
            for (int m = 0; m + 1 < end - start; ++m) rk4_step(fwd, seg[m], seg[m + 1], work[2], work[3], work[4]);
            for (int st = end - 1; st >= start; --st) {
                Field& un = seg[st - start];
                // forward stage arguments w1..w3 of step st (the step's result is discarded)
                rk4_step(fwd, un, work[1], work[2], work[3], work[4]);
                // adjoint step: stage arguments a0 = lam, a1..a3 = adjf[2..4]
                rk4_step(adj, *lam, *lamn, adjf[2], adjf[3], adjf[4]);
                const Field* args[4] = {lam, &adjf[2], &adjf[3], &adjf[4]};
                const Field* ws[4] = {&un, &work[2], &work[3], &work[4]};
                constexpr double bf[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
                for (int s = 0; s < 4; ++s) speed_gradient(*ws[3 - s], *args[s], dt * bf[s]);
                std::swap(lam, lamn);
            }
        }
        download(*lam, 0, grad_phi0);
        download(*lam, 1, grad_pi0);
        if (grad_c) {
            download(g, 0, grad_c);
            sync();
            for (long long q = 0; q < ncell; ++q) grad_c[q] *= 2.0 * c[q];
        }
        sync();
        return loss;
    }

    /// Tangent-linear run: (dphi_T, dpi_T) for the perturbation (dphi0, dpi0, dc) of (phi0, pi0, c).
    void tangent(const double* phi0, const double* pi0, const double* c, const double* dphi0, const double* dpi0,
                 const double* dc, int nsteps, double* dphiT, double* dpiT) {
        while (int(tanf.size()) < 5) tanf.emplace_back(n, G, NCT);
        std::vector<double> host(size_t(ncell) * NCT);
        for (long long q = 0; q < ncell; ++q) {
            host[q] = phi0[q];
            host[ncell + q] = pi0[q];
            host[2 * ncell + q] = c[q] * c[q];
            host[3 * ncell + q] = dphi0 ? dphi0[q] : 0.0;
            host[4 * ncell + q] = dpi0 ? dpi0[q] : 0.0;
            host[5 * ncell + q] = dc ? 2.0 * c[q] * dc[q] : 0.0;
        }
        upload_raw(tanf[0], host.data());
        Field* a = &tanf[0];
        Field* b = &tanf[1];
        for (int s = 0; s < nsteps; ++s) {
            rk4_step(tan, *a, *b, tanf[2], tanf[3], tanf[4]);
            std::swap(a, b);
        }
        download(*a, 3, dphiT);
        download(*a, 4, dpiT);
        sync();
    }

  private:
    int sm_count() const { return ts_context_sm_count(ctx); }
    void sync() { treesap_b200::cuda_check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize"); }

    void upload_raw(Field& f, const double* host) {
        const auto& L = f.layout();
        treesap_b200::cuda_check(cudaMemcpyAsync(staging, host, sizeof(double) * size_t(ncell) * L.nc,
                                                 cudaMemcpyHostToDevice, stream()),
                                 "cudaMemcpyAsync(upload)");
        treesap_b200::launch_pack(f.data(), L, staging, 0, sm_count(), stream());
        sync(); // the host buffer may go away
    }
    void upload_state(Field& f, const double* phi0, const double* pi0, const double* c) {
        std::vector<double> host(size_t(ncell) * NC);
        for (long long q = 0; q < ncell; ++q) {
            host[q] = phi0[q];
            host[ncell + q] = pi0 ? pi0[q] : 0.0;
            host[2 * ncell + q] = c[q] * c[q];
        }
        upload_raw(f, host.data());
    }
    /// Component `comp` of f's valid cells to the host (null: skipped).
    void download(const Field& f, int comp, double* host) {
        if (!host) return;
        const auto& L = f.layout();
        treesap_b200::launch_pack(f.data(), L, staging, 1, sm_count(), stream());
        treesap_b200::cuda_check(cudaMemcpyAsync(host, staging + size_t(comp) * ncell, sizeof(double) * size_t(ncell),
                                                 cudaMemcpyDeviceToHost, stream()),
                                 "cudaMemcpyAsync(download)");
        sync();
    }
    void copy(Field& dst, const Field& src) {
        treesap_b200::cuda_check(cudaMemcpyAsync(dst.data(), src.data(), size_t(src.layout().bytes()),
                                                 cudaMemcpyDeviceToDevice, stream()),
                                 "cudaMemcpyAsync(copy)");
    }
    void fill(Field& f) {
        // periodic images only: the domain is periodic in every direction
        treesap_b200::launch_ghost_fill(f.data(), f.layout(), geom, NoOpBC<NCT, G>{}, nullptr, 0.0,
                                        treesap_b200::GhostMode::Functor, sm_count(), stream());
    }

    template <class RHS, class Epi>
    void stage(const RHS& rhs, const Field& in, const typename Epi::Params& ep) {
        using Cfg = std::conditional_t<RHS::ncomp == NCT, TileT, Tile>;
        using Launcher = treesap_b200::StageLauncher<Cfg, RHS, Epi>;
        const auto& L = in.layout();
        const auto shape = Launcher::shape(L, sm_count());
        const CUtensorMap& tm = tmaps.get(in.data(), L, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
        const treesap_b200::CentreMaps cm = Launcher::centre_maps(
            [this](const void* b, const treesap_b200::Layout& Lc, int dtype, int bx, int by) -> const CUtensorMap& {
                return tmaps.get(b, Lc, dtype, bx, by);
            },
            ep, shape);
        treesap_b200::StageParams<double> sp{};
        sp.in = in.data();
        sp.L = L;
        sp.geom = geom;
        sp.time = 0.0;
        sp.err = ts_context_error_word(ctx);
        Launcher::launch(tm, cm, sp, rhs, ep, shape, stream());
    }

    /// One RK4 step u -> un with the stage arguments kept in w1, w2, w3 (the reference's
    /// register scheme, SingleLevelRK4Integrator.hpp:139-155, with three argument buffers).
    template <class RHS> void rk4_step(const RHS& rhs, Field& u, Field& un, Field& w1, Field& w2, Field& w3) {
        using namespace treesap_b200;
        constexpr double af[4] = {0.0, 0.5, 0.5, 1.0};
        constexpr double bf[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
        const Layout& L = u.layout();
        fill(u);
        stage<RHS, EpiRK4<0>>(rhs, u, {un.data(), w1.data(), u.data(), L, dt * bf[0], dt * af[1]});
        fill(w1);
        stage<RHS, EpiRK4<1>>(rhs, w1, {un.data(), w2.data(), u.data(), L, dt * bf[1], dt * af[2]});
        fill(w2);
        stage<RHS, EpiRK4<2>>(rhs, w2, {un.data(), w3.data(), u.data(), L, dt * bf[2], dt * af[3]});
        fill(w3);
        stage<RHS, EpiRK4<3>>(rhs, w3, {un.data(), nullptr, u.data(), L, dt * bf[3], 0.0});
    }

    /// g += b * a_pi * D w_phi (w has its ghost cells filled).
    void speed_gradient(const Field& w, const Field& a, double b) {
        stage<Lap, treesap_b200::EpiSpeedGradient>(Lap{}, w, {g.data(), a.data(), g.layout(), b});
    }

    ts_context* ctx;
    amrex::GeometryData geom;
    double dt;
    int every;
    int n[3] = {0, 0, 0};
    long long ncell = 0;
    Fwd fwd{};
    Adj adj{};
    Tan tan{};
    std::vector<Field> work, adjf, ckpt, seg, tanf;
    Field g;
    double* staging = nullptr;
    treesap_b200::TensorMapCache tmaps;
};

} // namespace treesap
