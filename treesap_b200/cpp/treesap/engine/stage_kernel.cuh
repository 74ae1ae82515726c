// treesap-b200 engine: the fused RK/Euler stage kernel.
//
// One launch evaluates one stage of the integrator over the whole box. The grid is
// (x-y tiles) x (z chunks), z-major: CTA b owns tile b % ntiles and z chunk b / ntiles, so the
// CTAs resident at any time hold neighbouring tiles at the same z and their halo re-reads hit
// in L2. A CTA has TY consumer warps (one 32-cell x row each, TY <= TYMAX chosen at launch) and
// one producer warp. Per z plane:
//
//   * the producer warp's elected lane copies the plane's tile plus its ghost halo, all
//     components, with one TMA load (cp.async.bulk.tensor.4d, no multicast; box
//     (TX+2*XH) x (TY+2G) x 1 x NC, zero fill outside the array) into a ring of R shared-memory
//     slots. Slot s has a `full` mbarrier (TMA transaction count) and an `empty` mbarrier
//     (one arrival per consumer warp); the producer refills a slot once every consumer warp
//     has released it, running up to R - G - 1 planes ahead of the computation.
//   * each consumer thread keeps its column's values at z-G .. z+G in a register queue,
//     shifted once per plane and fed from the newest plane.
//   * the user's RHS functor is called once per component, in component order, on an Array4
//     whose StencilView resolves every access at compile time: same-z offsets to the
//     shared-memory plane, same-column offsets to the register queue, anything else
//     (mixed x-z / y-z derivatives) to global memory.
//   * an epilogue policy combines the stage values with centre operands loaded one plane
//     ahead (register double buffer) and stores the results with coalesced stores.
//
// No CTA-wide barrier in the plane loop: warps proceed independently, bounded only by the
// ring. Every wait is bounded (ptx.cuh); on a timeout the kernel records an error bit, lets
// in-flight copies land and returns.
//
// Ring bookkeeping (per chunk, plane index it = 0 .. NP-1, z = z0 - G + it): plane it feeds the
// queue at iteration it and, when z0 <= z < z1, the x-y stencil taps at iteration it + G. After
// iteration it a consumer warp has released planes [0, released(it)):
//   released(it) = it + 1 (it < G),  G (G <= it < 2G),  it - G + 1 (it >= 2G),  NP (last).
#pragma once

#include <AMReX.H>
#include <cuda.h>

#include <cmath>
#include <cuda_runtime.h>

#include "../util/static_for.hpp"
#include "field.hpp"
#include "ptx.cuh"

namespace treesap_b200 {

template <int TX_, int TYMAX_, int G_, int NC_, typename T_, int P_ = 2, int MINB_ = 2> struct TileCfg {
    using T = T_;
    static constexpr int TX = TX_, TYMAX = TYMAX_, G = G_, NC = NC_, P = P_;
    static constexpr int MIN_BLOCKS = MINB_; // resident CTAs per SM the register budget is sized for
    static constexpr int A = 16 / int(sizeof(T));   // elements per 16 bytes
    static constexpr int XH = (G + A - 1) / A * A;  // x halo width in shared memory (16-byte aligned)
    static constexpr int BX = TX + 2 * XH;
    static constexpr int BYMAX = TYMAX + 2 * G;
    static constexpr int PLANE_MAX = NC * BYMAX * BX; // elements per slot (at TYMAX)
    static constexpr int R = G + 1 + P;               // ring slots
    static constexpr int THREADS = TX * TYMAX + 32;   // consumer warps + one producer warp
    static constexpr int SLOT_BYTES = (PLANE_MAX * int(sizeof(T)) + 127) / 128 * 128;
    static constexpr int SMEM = R * SLOT_BYTES + 16 * R;
    static_assert(TX == 32, "one warp per tile row");
    static_assert(BX <= 256 && BYMAX <= 256 && NC <= 256, "TMA box dimensions are limited to 256");
    static_assert(THREADS <= 1024, "too many threads");
};

/// Launch-invariant stage inputs.
template <typename T> struct StageParams {
    const T* in;              // stencil input field (global fallback for mixed x-z / y-z taps)
    Layout L;                 // its layout
    amrex::GeometryData geom; // passed to the RHS
    double time;              // stage time t + c_s dt
    int ntx, nty;             // tiles in x and y
    int ty;                   // tile height (rows = consumer warps), <= TYMAX
    int zchunk;               // planes per z chunk
    int* err;                 // device error word
};

template <class Cfg, class RHS, class Epi>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MIN_BLOCKS)
    stage_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams<typename Cfg::T> sp, const RHS rhs,
                 const typename Epi::Params ep) {
    using T = typename Cfg::T;
    constexpr int G = Cfg::G, NC = Cfg::NC, TX = Cfg::TX, BX = Cfg::BX, R = Cfg::R, XH = Cfg::XH;
    constexpr int SLOT = Cfg::SLOT_BYTES / int(sizeof(T));

    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* ring = reinterpret_cast<T*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + R * Cfg::SLOT_BYTES);
    uint64_t* empty = full + R;

    const int TY = sp.ty;
    const int BY = TY + 2 * G;
    const int PNS = BY * BX; // component stride inside a slot
    const int ntiles = sp.ntx * sp.nty;
    const int tile = blockIdx.x % ntiles;
    const int z0 = (blockIdx.x / ntiles) * sp.zchunk;
    const int z1 = min(sp.L.n[2], z0 + sp.zchunk);
    if (z0 >= z1) return;
    const int NP = (z1 - z0) + 2 * G; // planes streamed: z0 - G .. z1 - 1 + G
    const int x0 = (tile % sp.ntx) * TX, y0 = (tile / sp.ntx) * TY;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < R; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], uint32_t(TY));
        }
        ptx::fence_mbar_init();
    }
    __syncthreads();

    if (warp == TY) {
        // ---------------------------------------------------------------- producer warp
        if (lane == 0) {
            ptx::prefetch_tensor_map(&tmap);
            const uint32_t bytes = uint32_t(NC * BY * BX * int(sizeof(T)));
            int q = 0;
            for (; q < NP; ++q) {
                const int s = q % R;
                if (q >= R && !ptx::mbar_wait(&empty[s], uint32_t(((q / R) - 1) & 1), sp.err)) break;
                ptx::mbar_arrive_expect_tx(&full[s], bytes);
                // storage coordinates: x = x0 - XH + xoff (= x0), y = y0 - G + g (= y0), z = z0 - G + q + g
                ptx::tma_load_4d(ring + s * SLOT, &tmap, x0, y0, z0 + q, 0, &full[s]);
            }
            if (q < NP) {
                // a consumer warp stopped releasing slots: let the copies in flight land
                for (int r = (q > R ? q - R : 0); r < q; ++r)
                    ptx::mbar_wait(&full[r % R], uint32_t((r / R) & 1), nullptr, 100000000ull);
            }
        }
        return;
    }
    if (warp > TY) return;

    // -------------------------------------------------------------------- consumer warps
    // Register copies of everything the plane loop reads: values in kernel-parameter space are
    // not known to be loop-invariant, which would keep e.g. the stencils' 1/dx factors and the
    // functor's data inside the loop.
    const RHS f = rhs;
    const amrex::GeometryData geom = sp.geom;
    const Layout L = sp.L;
    const double time = sp.time;
    const typename Epi::Params epl = ep;

    const int tx = lane, ty = warp;
    const int i = x0 + tx, j = y0 + ty;
    const bool active = (i < L.n[0]) && (j < L.n[1]);
    const int coff = (ty + G) * BX + (tx + XH); // this thread's centre inside a slot

    T q[(2 * G + 1) * NC]; // register queue: q[(dk + G) * NC + c]
#pragma unroll
    for (int e = 0; e < (2 * G + 1) * NC; ++e) q[e] = T(0);

    using Pre = typename Epi::template Pre<NC>;
    Pre pre{};
    if (active) pre = Epi::template load<NC>(epl, i, j, z0);
    const T* in_col = sp.in + L.index(i, j, 0, 0); // global fallback: this column at z = 0
    const long long plane = L.px * L.py;

    int released = 0;
    for (int it = 0; it < NP; ++it) {
        const int s = it % R;
        if (!ptx::mbar_wait(&full[s], uint32_t((it / R) & 1), sp.err)) break;
        const T* slot = ring + s * SLOT;
#pragma unroll
        for (int e = 0; e < 2 * G * NC; ++e) q[e] = q[e + NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) q[2 * G * NC + c] = slot[c * PNS + coff];

        if (it >= 2 * G && active) {
            const int z = z0 - 2 * G + it;
            Pre pre_next{};
            if (z + 1 < z1) pre_next = Epi::template load<NC>(epl, i, j, z + 1);
            const T* ctr = ring + ((it - G) % R) * SLOT + coff;
            amrex::StencilView<T> view{ctr, q, in_col + z * plane, L.px, plane, L.comp_stride(), i, j, z, BX, PNS,
                                       G, NC};
            amrex::Array4<const T> arr = make_array4<const T>(sp.in, L);
            arr.view = &view;
            typename RHS::Workspace ws{};
            T kv[NC];
            const amrex::IntVect idx{i, j, z};
            treesap::static_for<NC>([&]<int c>() {
                kv[c] = static_cast<T>(f.template operator()<c>(idx, time, arr, geom, ws));
            });
            Epi::template apply<T, NC>(epl, kv, ctr, PNS, i, j, z, pre);
            pre = pre_next;
        }
        int rel = (it < G) ? it + 1 : (it < 2 * G ? G : it - G + 1);
        if (it == NP - 1) rel = NP;
        __syncwarp();
        if (lane == 0)
            for (int r = released; r < rel; ++r) ptx::mbar_arrive(&empty[r % R]);
        released = rel;
    }
}

// ------------------------------------------------------------------ epilogues
// Each policy: struct Params; struct Pre (centre operands loaded one plane ahead);
// static Pre load(params, i, j, z); template <T, NC> static void apply(params, k[NC], centre,
// pns, i, j, z, pre) where `centre` points at component 0 of the stencil input's centre in
// shared memory.

/// FP64 plain RK4 stage s with the reference's register scheme
/// (integrators/SingleLevelRK4Integrator.hpp:139-155):
///   s = 0:   acc = init + b k,  arg_next = init + a_next k   (the stencil input is init)
///   s = 1,2: acc += b k,        arg_next = init + a_next k
///   s = 3:   acc += b k
template <int STAGE> struct EpiRK4 {
    struct Params {
        double* acc;
        double* arg_next;
        const double* init;
        Layout L;
        double b, a_next;
    };
    template <int NC> struct Pre {
        double acc[NC];
        double init[NC];
    };
    template <int NC> static __device__ __forceinline__ Pre<NC> load(const Params& p, int i, int j, int z) {
        Pre<NC> r;
        if constexpr (STAGE > 0) {
            const long long o0 = p.L.index(i, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                r.acc[c] = __ldcs(p.acc + o0 + c * cs);
                if constexpr (STAGE < 3) r.init[c] = __ldg(p.init + o0 + c * cs);
            }
        }
        return r;
    }
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T* centre, int pns, int i,
                                                 int j, int z, const Pre<NC>& pre) {
        const long long o0 = p.L.index(i, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const long long o = o0 + c * cs;
            if constexpr (STAGE == 0) {
                const double u0 = centre[c * pns];
                __stcs(p.acc + o, u0 + p.b * k[c]);
                __stcs(p.arg_next + o, u0 + p.a_next * k[c]);
            } else {
                if constexpr (STAGE < 3) __stcs(p.arg_next + o, pre.init[c] + p.a_next * k[c]);
                __stcs(p.acc + o, pre.acc[c] + p.b * k[c]);
            }
        }
    }
};

/// Forward Euler (integrators/SingleLevelEulerIntegrator.hpp:77-84): new = old + dt k.
struct EpiEuler {
    struct Params {
        double* out;
        Layout L;
        double dt;
    };
    template <int NC> struct Pre {};
    template <int NC> static __device__ __forceinline__ Pre<NC> load(const Params&, int, int, int) { return {}; }
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T* centre, int pns, int i,
                                                 int j, int z, const Pre<NC>&) {
        const long long o0 = p.L.index(i, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) __stcs(p.out + o0 + c * cs, centre[c * pns] + p.dt * k[c]);
    }
};

/// FP32-stage RK4 for affine autonomous right-hand sides F(u) = L u + f0. The stage values
/// are carried as k0 plus differences d_s = k_s - k0, and every stencil of a full-magnitude
/// field runs in FP64 (a centred D2 of half-width 4 cancels ~1e6-fold, beyond FP32):
///   stage 0 (FP64 input u):   k0 = F(u);  u_p = u + dt k0                 -> k0 (FP64), u_p (FP64)
///   stage 1 (FP64 input k0):  d1 = dt/2 L k0                              -> d1 (FP32)
///   stage 2 (FP32 input d1):  d2 = d1 + dt/2 L d1        (= dt/2 L k1)     -> d2 (FP32)
///   stage 3 (FP32 input d2):  d3 = 2 d1 + dt L d2        (= dt L k2),
///                             u_new = u_p + dt/6 (2 d1 + 2 d2 + d3)  in FP64, in place
/// Algebraically u_new = u + dt/6 (k0 + 2 k1 + 2 k2 + k3) with k_s = F(u + a_s dt k_{s-1}).
struct EpiF32S0 {
    struct Params {
        double* k0;
        double* up;
        Layout Lu;
        double dt;
    };
    template <int NC> struct Pre {};
    template <int NC> static __device__ __forceinline__ Pre<NC> load(const Params&, int, int, int) { return {}; }
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T* centre, int pns, int i,
                                                 int j, int z, const Pre<NC>&) {
        const long long u0 = p.Lu.index(i, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            __stcs(p.k0 + u0 + c * us, double(k[c]));
            __stcs(p.up + u0 + c * us, double(centre[c * pns]) + p.dt * double(k[c]));
        }
    }
};

/// Stage 1 of the FP32-stage form: d1 = (dt/2) L k0 from the FP64 k0, stored FP32.
struct EpiF32S1 {
    struct Params {
        float* d1;
        Layout Lf;
        double a_dt;
    };
    template <int NC> struct Pre {};
    template <int NC> static __device__ __forceinline__ Pre<NC> load(const Params&, int, int, int) { return {}; }
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&lk)[NC], const T*, int, int i, int j,
                                                 int z, const Pre<NC>&) {
        const long long o0 = p.Lf.index(i, j, z, 0), cs = p.Lf.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) p.d1[o0 + c * cs] = static_cast<float>(p.a_dt * double(lk[c]));
    }
};

template <int STAGE> struct EpiF32Lin {
    struct Params {
        float* d_out;      // stages 1, 2: d1, d2
        const float* d1;   // stage 3
        double* u;         // stage 3: u_p in, u_new out (in place)
        Layout Lf, Lu;
        float a_dt;        // dt/2 (stages 1, 2), dt (stage 3)
        double dt;         // stage 3
    };
    template <int NC> struct Pre {
        float d1[NC];
        double up[NC];
    };
    template <int NC> static __device__ __forceinline__ Pre<NC> load(const Params& p, int i, int j, int z) {
        Pre<NC> r;
        if constexpr (STAGE == 3) {
            const long long o0 = p.Lf.index(i, j, z, 0), cs = p.Lf.comp_stride();
            const long long u0 = p.Lu.index(i, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                r.d1[c] = __ldcs(p.d1 + o0 + c * cs);
                r.up[c] = __ldcs(p.u + u0 + c * us);
            }
        }
        return r;
    }
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&lk)[NC], const T* centre, int pns, int i,
                                                 int j, int z, const Pre<NC>& pre) {
        const long long o0 = p.Lf.index(i, j, z, 0), cs = p.Lf.comp_stride();
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < NC; ++c) p.d_out[o0 + c * cs] = p.a_dt * lk[c];
        } else if constexpr (STAGE == 2) {
#pragma unroll
            for (int c = 0; c < NC; ++c) p.d_out[o0 + c * cs] = centre[c * pns] + p.a_dt * lk[c];
        } else {
            const long long u0 = p.Lu.index(i, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const float d1 = pre.d1[c], d2 = centre[c * pns];
                const float d3 = 2.0f * d1 + p.a_dt * lk[c];
                const double sum = 2.0 * double(d1) + 2.0 * double(d2) + double(d3);
                __stcs(p.u + u0 + c * us, pre.up[c] + (p.dt / 6.0) * sum);
            }
        }
    }
};

// ------------------------------------------------------------------ host launch
struct LaunchShape {
    int grid = 0;
    int ntx = 0, nty = 0, ty = 0;
    int nchunks = 0, zchunk = 0;
};

/// z-major grid: tiles of 32 x ty cells, the z extent split into `nchunks` chunks so that the
/// grid fills the resident CTA slots without chunks shorter than 4G planes (each chunk pays a
/// 2G-plane warm-up).
template <class Cfg> LaunchShape make_shape(const Layout& L, int slots, int ty, int nchunks = 0) {
    LaunchShape s;
    s.ty = ty;
    s.ntx = (L.n[0] + Cfg::TX - 1) / Cfg::TX;
    s.nty = (L.n[1] + ty - 1) / ty;
    const int ntiles = s.ntx * s.nty;
    if (nchunks <= 0) {
        nchunks = slots / ntiles;
        const int min_chunk = 4 * Cfg::G > 8 ? 4 * Cfg::G : 8;
        const int max_chunks = L.n[2] / min_chunk > 1 ? L.n[2] / min_chunk : 1;
        if (nchunks > max_chunks) nchunks = max_chunks;
        if (nchunks < 1) nchunks = 1;
    }
    s.zchunk = (L.n[2] + nchunks - 1) / nchunks;
    s.nchunks = (L.n[2] + s.zchunk - 1) / s.zchunk;
    s.grid = ntiles * s.nchunks;
    return s;
}

/// Tile height for a given width in x: the largest ty <= TYMAX whose tile count fills the SMs
/// most evenly (fraction of busy slot-time in the last wave), ties to the taller tile.
template <class Cfg> int choose_ty(const Layout& L, int slots) {
    int best = Cfg::TYMAX;
    double best_eff = -1.0;
    for (int ty = Cfg::TYMAX; ty >= (Cfg::TYMAX + 1) / 2; --ty) {
        const LaunchShape s = make_shape<Cfg>(L, slots, ty);
        const double waves = double(s.grid) / slots;
        const double eff = waves / std::ceil(waves) * (double(ty) / Cfg::TYMAX > 0.75 ? 1.0 : 0.95);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = ty;
        }
    }
    return best;
}

template <class Cfg, class RHS, class Epi> struct StageLauncher {
    static auto kernel() { return &stage_kernel<Cfg, RHS, Epi>; }
    /// Resident CTAs per SM for this instantiation (sets the dynamic shared-memory limit once per device).
    static int occupancy() {
        static int occ[64] = {0};
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev < 0 || dev >= 64) dev = 0;
        if (occ[dev] == 0) {
            cuda_check(cudaFuncSetAttribute(kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM),
                       "cudaFuncSetAttribute(smem)");
            int nb = 0;
            cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel(), Cfg::THREADS, Cfg::SMEM),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            occ[dev] = nb > 0 ? nb : 1;
        }
        return occ[dev];
    }
    /// Launch shape for a layout; `ty` <= 0 picks the tile height, `nchunks` <= 0 the z split.
    static LaunchShape shape(const Layout& L, int sm_count, int ty = 0, int nchunks = 0) {
        const int slots = occupancy() * sm_count;
        if (ty <= 0 || ty > Cfg::TYMAX) ty = choose_ty<Cfg>(L, slots);
        return make_shape<Cfg>(L, slots, ty, nchunks);
    }
    /// The TMA box of a launch shape: (TX + 2 XH) x (ty + 2G).
    static int box_x() { return Cfg::BX; }
    static int box_y(const LaunchShape& s) { return s.ty + 2 * Cfg::G; }
    static void launch(const CUtensorMap& tmap, StageParams<typename Cfg::T> sp, const RHS& rhs,
                       const typename Epi::Params& ep, const LaunchShape& s, cudaStream_t stream) {
        sp.ntx = s.ntx;
        sp.nty = s.nty;
        sp.ty = s.ty;
        sp.zchunk = s.zchunk;
        const int threads = 32 * s.ty + 32;
        stage_kernel<Cfg, RHS, Epi><<<s.grid, threads, Cfg::SMEM, stream>>>(tmap, sp, rhs, ep);
        cuda_check(cudaGetLastError(), "stage_kernel launch");
    }
};

} // namespace treesap_b200
