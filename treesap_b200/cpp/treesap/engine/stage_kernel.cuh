// treesap-b200 engine: the fused RK/Euler stage kernel.
//
// One launch evaluates one stage of the integrator over the whole box. Each CTA owns an
// x-y tile of TX x TY cells (one thread per cell, a warp per x row) and marches along z
// over one or two contiguous z segments (a balanced split of tile-major work across a
// grid sized to the resident CTA slots). Per z plane:
//
//   * TMA (cp.async.bulk.tensor.4d, no multicast) copies the plane's tile plus its ghost
//     halo, all components, into a ring of R shared-memory slots (box (TX+2*XH) x (TY+2G) x 1 x NC,
//     zero fill outside the array); one mbarrier per slot, a single elected producer thread.
//   * Each thread keeps its column's values at z-G .. z+G in registers (a queue shifted
//     once per plane and fed from the newest plane in shared memory).
//   * The user's RHS functor is called once per component, in component order, on an
//     Array4 whose StencilView resolves every access at compile time: same-z offsets to
//     the shared-memory plane, same-column offsets to the register queue, anything else
//     (mixed x-z / y-z derivatives) to global memory.
//   * An epilogue policy combines the stage values with the register state and stores
//     the results (stage accumulator, next-stage argument, ...) with coalesced stores.
//
// Ring bookkeeping: the planes of a segment are streamed in order; plane `it` (local
// index, z = z_begin - G + it) is consumed by the queue at iteration it and, when it
// lies in the segment, by the x-y stencil taps at iteration it + G. A slot is handed
// back to the producer after a CTA barrier once its plane is no longer needed, so the
// loads run up to R - G - 1 planes ahead of the computation.
#pragma once

#include <AMReX.H>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../util/static_for.hpp"
#include "field.hpp"
#include "ptx.cuh"

namespace treesap_b200 {

template <int TX_, int TY_, int G_, int NC_, typename T_, int P_ = 2> struct TileCfg {
    using T = T_;
    static constexpr int TX = TX_, TY = TY_, G = G_, NC = NC_, P = P_;
    static constexpr int A = 16 / int(sizeof(T)); // elements per 16 bytes
    static constexpr int XH = (G + A - 1) / A * A; // x halo width in shared memory (16-byte aligned)
    static constexpr int BX = TX + 2 * XH;
    static constexpr int BY = TY + 2 * G;
    static constexpr int PLANE = NC * BY * BX; // elements per slot
    static constexpr int R = G + 1 + P;        // ring slots
    static constexpr int THREADS = TX * TY;
    static constexpr int SLOT_BYTES = (PLANE * int(sizeof(T)) + 127) / 128 * 128;
    static constexpr int SMEM = R * SLOT_BYTES + 8 * R;
    static_assert(TX % A == 0, "tile width must be a multiple of 16 bytes");
    static_assert(BX <= 256 && BY <= 256 && NC <= 256, "TMA box dimensions are limited to 256");
    static_assert(THREADS <= 1024, "too many threads");
};

/// Launch-invariant stage inputs.
template <typename T> struct StageParams {
    const T* in;               // stencil input field (global fallback for mixed x-z / y-z taps)
    Layout L;                  // its layout
    amrex::GeometryData geom;  // passed to the RHS
    double time;               // stage time t + c_s dt
    int ntx, nty;              // tiles in x and y
    long long work;            // ntx * nty * n[2] plane-cells of work
    int* err;                  // device error word
};

template <class Cfg, class RHS, class Epi>
__global__ void __launch_bounds__(Cfg::THREADS)
    stage_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams<typename Cfg::T> sp, const RHS rhs,
                 const typename Epi::Params ep) {
    using T = typename Cfg::T;
    constexpr int G = Cfg::G, NC = Cfg::NC, TX = Cfg::TX, BX = Cfg::BX, BY = Cfg::BY, R = Cfg::R, XH = Cfg::XH;
    constexpr int SLOT = Cfg::SLOT_BYTES / int(sizeof(T));
    constexpr int PNS = BY * BX; // component stride inside a slot

    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* ring = reinterpret_cast<T*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + R * Cfg::SLOT_BYTES);

    const int nz = sp.L.n[2];
    const long long W = sp.work;
    const long long wb = W * blockIdx.x / gridDim.x, we = W * (blockIdx.x + 1) / gridDim.x;
    if (wb >= we) return;

    // Segments of this CTA: maximal runs of [wb, we) inside one tile column.
    // Plane stream: segment by segment, planes z_b - G .. z_e - 1 + G.
    auto seg_tile = [&](long long w) { return int(w / nz); };
    long long total_planes = 0;
    for (long long w = wb; w < we;) {
        const long long wend = (w / nz + 1) * nz < we ? (w / nz + 1) * nz : we;
        total_planes += (wend - w) + 2 * G;
        w = wend;
    }

    if (threadIdx.x == 0) {
        ptx::prefetch_tensor_map(&tmap);
        for (int s = 0; s < R; ++s) ptx::mbar_init(&full[s], 1);
        ptx::fence_mbar_init();
    }
    __syncthreads();

    // Producer state (thread 0 only): the stream is re-derived from (segment, local index).
    long long issued = 0;
    long long prod_w = wb; // segment cursor of the producer
    int prod_it = 0;       // local plane index inside the producer's segment
    auto issue_upto = [&](long long limit) {
        while (issued < limit && issued < total_planes) {
            const int tile = seg_tile(prod_w);
            const int zb = int(prod_w % nz);
            const long long sege = ((prod_w / nz) + 1) * nz < we ? ((prod_w / nz) + 1) * nz : we;
            const int nplanes = int(sege - prod_w) + 2 * G;
            const int s = int(issued % R);
            const int x0 = (tile % sp.ntx) * TX, y0 = (tile / sp.ntx) * Cfg::TY;
            ptx::mbar_arrive_expect_tx(&full[s], uint32_t(Cfg::PLANE * sizeof(T)));
            // storage coordinates: x = x0 - XH + xoff (= x0), y = y0 - G + g (= y0), z = zb - G + it + g
            ptx::tma_load_4d(ring + s * SLOT, &tmap, x0, y0, zb + prod_it, 0, &full[s]);
            ++issued;
            if (++prod_it == nplanes) {
                prod_it = 0;
                prod_w = sege;
            }
        }
    };
    if (threadIdx.x == 0) issue_upto(R);

    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int coff = (ty + G) * BX + (tx + XH); // this thread's centre inside a slot

    T q[(2 * G + 1) * NC]; // register queue: q[(dk + G) * NC + c]
#pragma unroll
    for (int e = 0; e < (2 * G + 1) * NC; ++e) q[e] = T(0);

    long long consumed = 0; // planes fully released (slot handed back)
    long long streamed = 0; // planes consumed by the queue so far (global stream index)
    bool failed = false;

    for (long long w = wb; w < we && !failed;) {
        const int tile = seg_tile(w);
        const int zb = int(w % nz);
        const long long sege = ((w / nz) + 1) * nz < we ? ((w / nz) + 1) * nz : we;
        const int nplanes = int(sege - w) + 2 * G;
        const long long seg_base = streamed;
        const int i = (tile % sp.ntx) * TX + tx;
        const int j = (tile / sp.ntx) * Cfg::TY + ty;
        const bool active = (i < sp.L.n[0]) && (j < sp.L.n[1]);

        for (int it = 0; it < nplanes; ++it) {
            const long long gq = seg_base + it;
            const int s = int(gq % R);
            if (!ptx::mbar_wait(&full[s], uint32_t((gq / R) & 1), sp.err)) failed = true;
            if (!failed) {
                const T* slot = ring + s * SLOT;
#pragma unroll
                for (int e = 0; e < 2 * G * NC; ++e) q[e] = q[e + NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) q[2 * G * NC + c] = slot[c * PNS + coff];

                if (it >= 2 * G && active) {
                    const int z = zb - 2 * G + it;
                    const T* ctr = ring + int((gq - G) % R) * SLOT + coff;
                    amrex::StencilView<T> view{ctr,
                                               q,
                                               sp.in + sp.L.index(i, j, z, 0),
                                               sp.L.px,
                                               sp.L.px * sp.L.py,
                                               sp.L.comp_stride(),
                                               i,
                                               j,
                                               z,
                                               BX,
                                               PNS,
                                               G,
                                               NC};
                    amrex::Array4<const T> arr = make_array4<const T>(sp.in, sp.L);
                    arr.view = &view;
                    typename RHS::Workspace ws{};
                    T kv[NC];
                    const amrex::IntVect idx{i, j, z};
                    treesap::static_for<NC>([&]<int c>() {
                        kv[c] = static_cast<T>(rhs.template operator()<c>(idx, sp.time, arr, sp.geom, ws));
                    });
                    Epi::template apply<T, NC>(ep, kv, ctr, PNS, i, j, z);
                }
            }
            streamed = gq + 1;
            // release: planes below z_b are only queue inputs; planes inside the segment are
            // released after their x-y taps were used (G iterations after they arrived)
            long long released = seg_base + (it < G ? it + 1 : (it < 2 * G ? G : it - G + 1));
            if (it == nplanes - 1) released = seg_base + nplanes;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            if (threadIdx.x == 0) {
                ptx::fence_proxy_async_smem();
                consumed = released;
                issue_upto(consumed + R);
            }
        }
        w = sege;
    }

    if (failed && threadIdx.x == 0) {
        // Let copies still in flight land before the CTA's shared memory is released.
        for (long long gq = streamed; gq < issued; ++gq)
            ptx::mbar_wait(&full[int(gq % R)], uint32_t((gq / R) & 1), sp.err, 100000000ull);
    }
}

// ------------------------------------------------------------------ epilogues
// Each policy: struct Params; template <T, NC> static void apply(params, k[NC], centre, pns, i, j, z)
// where `centre` points at component 0 of the stencil input's centre in shared memory.

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
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T* centre, int pns, int i,
                                                 int j, int z) {
        const long long o0 = p.L.index(i, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const long long o = o0 + c * cs;
            if constexpr (STAGE == 0) {
                const double u0 = centre[c * pns];
                p.acc[o] = u0 + p.b * k[c];
                p.arg_next[o] = u0 + p.a_next * k[c];
            } else {
                const double a0 = p.acc[o];
                if constexpr (STAGE < 3) {
                    const double u0 = __ldg(p.init + o);
                    p.arg_next[o] = u0 + p.a_next * k[c];
                }
                p.acc[o] = a0 + p.b * k[c];
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
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T* centre, int pns, int i,
                                                 int j, int z) {
        const long long o0 = p.L.index(i, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) p.out[o0 + c * cs] = centre[c * pns] + p.dt * k[c];
    }
};

/// FP32-stage RK4 for affine autonomous right-hand sides F(u) = L u + f0.
///   stage 0 (FP64 input u):   k0 = F(u)                         -> k0 (FP32)
///   stage 1 (FP32 input k0):  k1 = k0 + (dt/2) L k0             -> k1
///   stage 2 (FP32 input k1):  k2 = k0 + (dt/2) L k1             -> k2
///   stage 3 (FP32 input k2):  k3 = k0 + dt L k2,
///                             u_new = u + dt/6 (k0 + 2 k1 + 2 k2 + k3)  in FP64
/// which is algebraically the classical RK4 step k_s = F(u + a_s dt k_{s-1}).
struct EpiF32S0 {
    struct Params {
        float* k0;
        Layout Lf;
    };
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[NC], const T*, int, int i, int j,
                                                 int z) {
        const long long o0 = p.Lf.index(i, j, z, 0), cs = p.Lf.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) p.k0[o0 + c * cs] = static_cast<float>(k[c]);
    }
};

template <int STAGE> struct EpiF32Lin {
    struct Params {
        float* k_out;       // stages 1, 2
        const float* k0;    // stages 2, 3
        const float* k1;    // stage 3
        const double* u_in; // stage 3: state at the start of the step
        double* u;          // stage 3: state at the end of the step
        Layout Lf, Lu;
        float a_dt;         // a_s dt
        double dt;          // stage 3
    };
    template <class T, int NC>
    static __device__ __forceinline__ void apply(const Params& p, const T (&lk)[NC], const T* centre, int pns, int i,
                                                 int j, int z) {
        const long long o0 = p.Lf.index(i, j, z, 0), cs = p.Lf.comp_stride();
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < NC; ++c) p.k_out[o0 + c * cs] = centre[c * pns] + p.a_dt * lk[c];
        } else if constexpr (STAGE == 2) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const long long o = o0 + c * cs;
                p.k_out[o] = __ldg(p.k0 + o) + p.a_dt * lk[c];
            }
        } else {
            const long long u0 = p.Lu.index(i, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const long long o = o0 + c * cs;
                const float k0 = __ldg(p.k0 + o), k1 = __ldg(p.k1 + o), k2 = centre[c * pns];
                const float k3 = k0 + p.a_dt * lk[c];
                const double sum = double(k0) + 2.0 * double(k1) + 2.0 * double(k2) + double(k3);
                p.u[u0 + c * us] = __ldg(p.u_in + u0 + c * us) + (p.dt / 6.0) * sum;
            }
        }
    }
};

// ------------------------------------------------------------------ host launch
struct LaunchShape {
    int grid = 0;
    int ntx = 0, nty = 0;
    long long work = 0;
};

/// Grid size: one CTA per resident slot (occupancy x SMs), but no CTA with less than
/// `min_planes` planes of work (short segments pay 2G warm-up planes each).
template <class Cfg> LaunchShape make_shape(const Layout& L, int slots) {
    LaunchShape s;
    s.ntx = (L.n[0] + Cfg::TX - 1) / Cfg::TX;
    s.nty = (L.n[1] + Cfg::TY - 1) / Cfg::TY;
    s.work = (long long)s.ntx * s.nty * L.n[2];
    const long long min_planes = 8 * Cfg::G > 16 ? 8 * Cfg::G : 16;
    long long g = (s.work + min_planes - 1) / min_planes;
    if (g > slots) g = slots;
    if (g < 1) g = 1;
    s.grid = int(g);
    return s;
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
    static void launch(const CUtensorMap& tmap, StageParams<typename Cfg::T> sp, const RHS& rhs,
                       const typename Epi::Params& ep, int sm_count, cudaStream_t stream) {
        const LaunchShape s = make_shape<Cfg>(sp.L, occupancy() * sm_count);
        sp.ntx = s.ntx;
        sp.nty = s.nty;
        sp.work = s.work;
        stage_kernel<Cfg, RHS, Epi><<<s.grid, Cfg::THREADS, Cfg::SMEM, stream>>>(tmap, sp, rhs, ep);
        cuda_check(cudaGetLastError(), "stage_kernel launch");
    }
};

} // namespace treesap_b200
