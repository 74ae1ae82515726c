// treesap-b200 engine: the fused RK/Euler stage kernel.
//
// One launch evaluates one stage of the integrator over the whole box. The grid is
// (x-y tiles) x (z chunks), z-major: CTA b owns tile b % ntiles and z chunk b / ntiles, so the
// CTAs resident at any time hold neighbouring tiles at the same z and their halo re-reads hit
// in L2. A CTA has TY consumer warps (CY rows of TX = 32 CX cells each, TY <= TYMAX chosen at
// launch) and one producer warp. Per z plane:
//
//   * the producer warp's elected lane copies the plane's tile plus its ghost halo, all
//     components, with one TMA load (cp.async.bulk.tensor.4d into this CTA only; box
//     (TX+2*XH) x (TY*CY+2G) x 1 x NC, zero fill outside the array) into a ring of R shared-memory
//     slots. When the plane is also a stencil centre plane of this CTA, the same slot receives
//     the epilogue's centre operands (the stage registers it reads at the centre cells, e.g.
//     the RK4 accumulator and initial state): one more TMA box (TX x TY*CY x 1 x NC) per operand
//     field, completing on the same barrier. Slot s has a `full` mbarrier (TMA transaction
//     count) and an `empty` mbarrier (one arrival per consumer warp); the producer refills a
//     slot once every consumer warp has released it, running up to R - G - 1 planes ahead of
//     the queue and R - 1 planes ahead of the centre computation.
//   * each consumer thread keeps its CX x CY columns' values at z-G .. z+G in a register
//     queue, shifted once per plane and fed from the newest plane. The CY rows of a thread
//     share their y taps (rows j0-G .. j0+CY-1+G), which the compiler loads once.
//   * the user's RHS functor is called once per component, in component order, on an Array4
//     whose StencilView resolves every access at compile time: same-z offsets to the
//     shared-memory plane, same-column offsets to the register queue, anything else
//     (mixed x-z / y-z derivatives) to global memory.
//   * an epilogue policy combines the stage values with the centre operands from shared memory
//     and stores the results with coalesced stores.
//
// No CTA-wide barrier in the plane loop: warps proceed independently, bounded only by the
// ring. Every wait is bounded (ptx.cuh); on a timeout the kernel records an error bit, lets
// in-flight copies land and returns.
//
// Ring bookkeeping (per chunk, plane index it = 0 .. NP-1, z = z0 - G + it): plane it feeds the
// queue at iteration it and, when z0 <= z < z1, the x-y stencil taps and the centre operands at
// iteration it + G. Each consumer warp releases plane p after iteration p (p < G) or p + G
// (p >= G), one plane per iteration; the producer refills a slot with plane q once plane q - R
// is released (R >= G + 2, so the newest plane never waits on a plane still in use).
#pragma once

#include <AMReX.H>
#include <cuda.h>

#include <cmath>
#include <cuda_runtime.h>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

#include "../util/static_for.hpp"
#include "field.hpp"
#include "ptx.cuh"

namespace treesap_b200 {

constexpr int align128(int b) { return (b + 127) / 128 * 128; }

/// Tile configuration of the stage kernel: CX cells per thread along x (a warp covers
/// TX = 32 CX cells of a row), CY rows per consumer warp, up to TYMAX consumer warps (a tile
/// is ty * CY rows high), ghost width G, NC components of type T, up to P planes of prefetch,
/// MINB resident CTAs per SM, U planes per iteration of the plane loop.
template <int CX_, int TYMAX_, int G_, int NC_, typename T_, int P_ = 2, int MINB_ = 2, int U_ = 1, int CY_ = 1,
          bool ROT_ = false, bool ZQ_ = true>
struct TileCfg {
    using T = T_;
    static constexpr int CX = CX_, TX = 32 * CX_, TYMAX = TYMAX_, G = G_, NC = NC_, P = P_, U = U_, CY = CY_;
    /// ZQ: z taps at the cell's column from a register queue of 2G + U planes fed by a ring that
    /// also streams the G halo planes above and below; !ZQ (many components, whose queue would
    /// not fit the registers): the ring streams only the centre planes and every tap off the
    /// centre plane is a global load (L1/L2).
    static constexpr bool ZQ = ZQ_;
    static constexpr int ZH = ZQ_ ? G_ : 0; // halo planes streamed below and above a z range
    /// Circular register queue: the plane loop is unrolled by the queue depth 2G + 1 so that
    /// every plane keeps its register slot (plane % (2G + 1)) instead of being shifted.
    static constexpr bool ROT = ROT_;
    static constexpr int MIN_BLOCKS = MINB_; // resident CTAs per SM the register and smem budgets are sized for
    static constexpr int A = 16 / int(sizeof(T));   // elements per 16 bytes
    static constexpr int XH = (G + A - 1) / A * A;  // x halo width in shared memory (16-byte aligned)
    static constexpr int BX = TX + 2 * XH;
    static constexpr int BYMAX = TYMAX * CY + 2 * G;
    static constexpr int PLANE_MAX = NC * BYMAX * BX;  // stencil elements per slot (at TYMAX)
    static constexpr int THREADS = 32 * TYMAX + 32;    // consumer warps + one producer warp
    static constexpr int STENCIL_BYTES = align128(PLANE_MAX * int(sizeof(T)));
    static constexpr int CBOX = NC * TYMAX * CY * TX;  // elements of one centre-operand box
    /// Dynamic shared memory per CTA when MIN_BLOCKS CTAs share an SM (228 KB per SM with 1 KB
    /// reserved per CTA; at most 227 KB for one CTA).
    static constexpr int SMEM_BUDGET = MINB_ == 1 ? 232448 : 233472 / MINB_ - 1024;
    /// Shared memory of a stencil ring of ZH + U + p slots and a centre-operand ring of U + p
    /// slots of `cslot` bytes (none when cslot = 0), with their mbarriers.
    static constexpr int smem_for(int p, int cslot) {
        return (ZH + U + p) * (STENCIL_BYTES + 16) + (cslot > 0 ? (U + p) * (cslot + 8) : 0);
    }
    /// Usable when even two FP64 centre-operand fields fit with one plane of prefetch.
    static constexpr bool fits = smem_for(1, 2 * align128(CBOX * 8)) <= SMEM_BUDGET;
    static_assert(CX == 1 || CX == 2, "one or two cells per thread along x");
    static_assert(U == 1 || U == 2, "one or two planes per iteration");
    static_assert(CY >= 1 && CY <= 4, "one to four rows per consumer warp");
    static_assert(!ROT || U == 1, "the circular queue takes one plane per iteration");
    static_assert(ZQ || (U == 1 && !ROT), "without the register queue: one plane per iteration, no rotation");
    static_assert(BX <= 256 && BYMAX <= 256 && NC <= 256, "TMA box dimensions are limited to 256");
    static_assert(THREADS <= 1024, "too many threads");
};

/// Shared-memory rings of one (tile configuration, epilogue) pair:
///   * the stencil ring, R = G + U + P slots, each one stencil plane ([comp][y][x], TY CY + 2G
///     rows of BX), with a `full` and an `empty` mbarrier per slot;
///   * the centre-operand ring, RC slots (none without centre operands), each the epilogue's
///     centre-operand boxes of one centre plane ([comp][y][x], TY CY rows of TX per field,
///     128-byte aligned), with an `empty` mbarrier per slot. The boxes of centre plane c are
///     copied together with (and complete on the `full` barrier of) stencil plane c + G, the
///     newest plane of the iteration that computes centre plane c.
/// Static layout (circular register queue, one plane per iteration): R equals the queue depth
/// QL = 2G + 1 (P = G), so that in the plane loop, which is unrolled QL times, every stencil
/// slot is a compile-time constant (single-item launches) and no slot counter is carried from
/// plane to plane; the same holds for the centre ring when its size divides QL. Otherwise P is
/// the configuration's prefetch depth, reduced until both rings fit the budget. The centre ring
/// has up to U + P slots (as many as fit); fewer cap the prefetch depth at RC - 1 planes.
template <class Cfg, class Epi> struct Ring {
    using C0 = typename Epi::C0;
    using C1 = typename Epi::C1;
    static constexpr int NCEN = Epi::kCentre;
    static_assert(NCEN >= 0 && NCEN <= 2, "at most two centre-operand fields");
    static constexpr int SSLOT = Cfg::STENCIL_BYTES;
    static constexpr int C0_OFF = 0; // within a centre slot
    static constexpr int C1_OFF = NCEN > 0 ? align128(Cfg::CBOX * int(sizeof(C0))) : 0;
    static constexpr int CSLOT = NCEN > 1 ? C1_OFF + align128(Cfg::CBOX * int(sizeof(C1))) : C1_OFF;
    static constexpr int QL = 2 * Cfg::ZH + Cfg::U;
    static constexpr int bytes(int r, int rc) { return r * (SSLOT + 16) + rc * (CSLOT + 8); }
    /// Static layout: circular queue, one plane per iteration, and R = QL stencil slots fit.
    static constexpr bool kStatic = Cfg::ROT && Cfg::U == 1 && Cfg::ZQ && bytes(QL, NCEN > 0 ? 1 : 0) <= Cfg::SMEM_BUDGET;
    static constexpr int P = kStatic ? QL - Cfg::ZH - Cfg::U : [] {
        int p = Cfg::P;
        while (p > 1 && Cfg::smem_for(p, CSLOT) > Cfg::SMEM_BUDGET) --p;
        return p;
    }();
    static constexpr int R = Cfg::ZH + Cfg::U + P;
    /// Centre ring: QL slots in the static layout when they fit (compile-time slots), else up to
    /// U + P slots, as many as fit beside the stencil ring.
    static constexpr int RC = [] {
        if (NCEN > 0 && kStatic && bytes(R, QL) <= Cfg::SMEM_BUDGET) return QL;
        int rc = NCEN > 0 ? Cfg::U + P : 0;
        while (rc > 1 && bytes(R, rc) > Cfg::SMEM_BUDGET) --rc;
        return rc;
    }();
    /// Centre-ring slots are compile-time constants too when RC divides QL.
    static constexpr bool kStaticCentre = kStatic && (RC == 0 || QL % RC == 0);
    static constexpr int CRING_OFF = R * SSLOT;             // centre ring
    static constexpr int BAR_OFF = CRING_OFF + RC * CSLOT;  // full[R], empty[R], cempty[RC]
    static constexpr int SMEM = BAR_OFF + 8 * (2 * R + RC);
    static_assert(!kStatic || R == QL, "static ring layout");
    static_assert(bytes(R, RC) <= Cfg::SMEM_BUDGET, "shared-memory rings too large for this tile configuration");
};

/// Launch-invariant stage inputs.
template <typename T> struct StageParams {
    const T* in;              // stencil input field (global fallback for mixed x-z / y-z taps)
    Layout L;                 // its layout
    amrex::GeometryData geom; // passed to the RHS
    double time;              // stage time t + c_s dt
    int ntx, nty;             // tiles in x and y
    int ty;                   // consumer warps (a tile is ty * CY rows high), <= TYMAX
    int zchunk;               // planes per z chunk
    int* err;                 // device error word
    unsigned long long wait_ns = kWaitLimitNs; // bound of every mbarrier wait of the launch
    int skip_plane = -1; // injected fault: the producer skips the copy of this plane of every item
    int zoff = 0;        // global z index of the input's plane 0 (a z slab of a larger domain)
};

/// TMA descriptors of the centre-operand fields (box TX x ty CY x 1 x NC) and the storage
/// coordinates of cell (0, 0, 0) in each (x = xoff, y = z = ngrow).
struct alignas(64) CentreMaps {
    CUtensorMap map[2];
    int x[2], y[2], z[2];
};

/// What an epilogue reads at its centre cell: component c of operand field k is ck[c * cps].
template <class C0, class C1> struct CentreOps {
    const C0* c0;
    const C1* c1;
    int cps;
};

/// Host-side description of one centre-operand field.
struct CentreSrc {
    const void* base;
    Layout L;
    int dtype; // ts_dtype
};

/// Slot and completion parity of a plane in a ring of R slots, advanced plane by plane.
struct RingPos {
    int s = 0;
    uint32_t ph = 0;
    __device__ __forceinline__ void next(int R) {
        if (++s == R) {
            s = 0;
            ph ^= 1u;
        }
    }
};

/// CX consecutive elements from shared memory (one vector load for CX = 2; 2 CX-element alignment).
template <int CX, class V> __device__ __forceinline__ void lds(const V* p, V (&out)[CX]) {
    if constexpr (CX == 2 && sizeof(V) == 8) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        out[0] = v.x;
        out[1] = v.y;
    } else if constexpr (CX == 2 && sizeof(V) == 4) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        out[0] = v.x;
        out[1] = v.y;
    } else {
#pragma unroll
        for (int e = 0; e < CX; ++e) out[e] = p[e];
    }
}

/// Streaming store of CX consecutive cells, skipping inactive ones (one vector store when all
/// CX are active; the address of cell 0 is aligned to CX elements).
template <int CX, class V>
__device__ __forceinline__ void stcs(V* p, const V (&v)[CX], const bool (&act)[CX]) {
    if constexpr (CX == 2) {
        if (act[0] && act[1]) {
            if constexpr (sizeof(V) == 8)
                __stcs(reinterpret_cast<double2*>(p), make_double2(v[0], v[1]));
            else
                __stcs(reinterpret_cast<float2*>(p), make_float2(v[0], v[1]));
            return;
        }
    }
#pragma unroll
    for (int e = 0; e < CX; ++e)
        if (act[e]) __stcs(p + e, v[e]);
}

/// The RHS functor for every component of one cell, in component order, on one workspace
/// (SingleLevelRK4Integrator.hpp:139-155). A fold rather than a lambda: a lambda that the
/// compiler declines to inline (many components) would force the register queue that the
/// Array4's view points at into local memory.
template <class RHS, class T, int NC, int... C>
__device__ __forceinline__ void eval_components(const RHS& f, T (&kv)[NC], const amrex::IntVect& idx, double time,
                                                const amrex::Array4<const T>& arr, const amrex::GeometryData& geom,
                                                typename RHS::Workspace& ws, std::integer_sequence<int, C...>) {
    ((kv[C] = static_cast<T>(f.template operator()<C>(idx, time, arr, geom, ws))), ...);
}

/// The stage values of one cell: the RHS on an Array4 whose accesses the view resolves.
template <class RHS, class T, int NC>
__device__ __forceinline__ void eval_cell(const RHS& f, T (&kv)[NC], const amrex::StencilView<T>& view, const T* in,
                                          const Layout& L, const amrex::IntVect& idx, double time,
                                          const amrex::GeometryData& geom, int zoff) {
    amrex::Array4<const T> arr = make_array4<const T>(in, L, zoff);
    arr.view = &view;
    typename RHS::Workspace ws{};
    eval_components(f, kv, idx, time, arr, geom, ws, std::make_integer_sequence<int, NC>{});
}

/// One unit of work of a CTA: the tile at (x0, y0) of instance `inst`, planes z0 .. z1-1.
struct ItemBox {
    int inst, x0, y0, z0, z1;
};

/// Work source of a single-box launch: one item per CTA (tile blockIdx % ntiles, z chunk
/// blockIdx / ntiles), everything else in kernel-parameter space.
template <class Cfg, class RHS, class Epi> struct SingleSource {
    using T = typename Cfg::T;
    static constexpr bool kSingleItem = true; // at most one item per CTA: rings start at slot 0
    const CUtensorMap* tmap;
    const CentreMaps* cmaps;
    const StageParams<T>* sp;
    const RHS* rhs;
    const typename Epi::Params* ep;
    __device__ __forceinline__ int ty() const { return sp->ty; }
    __device__ __forceinline__ int* err() const { return sp->err; }
    __device__ __forceinline__ ItemBox first() const {
        const int ntiles = sp->ntx * sp->nty;
        const int tile = blockIdx.x % ntiles;
        const int z0 = (blockIdx.x / ntiles) * sp->zchunk;
        return {0, (tile % sp->ntx) * Cfg::TX, (tile / sp->ntx) * sp->ty * Cfg::CY, z0,
                min(sp->L.n[2], z0 + sp->zchunk)};
    }
    __device__ __forceinline__ int count() const {
        const ItemBox b = first();
        return b.z0 < b.z1 ? 1 : 0;
    }
    __device__ __forceinline__ ItemBox item(int) const { return first(); }
    __device__ __forceinline__ const CUtensorMap* stencil_map(int) const { return tmap; }
    __device__ __forceinline__ const CentreMaps& centre_maps(int) const { return *cmaps; }
    __device__ __forceinline__ const StageParams<T>& params(int) const { return *sp; }
    __device__ __forceinline__ const RHS& rhs_of(int) const { return *rhs; }
    __device__ __forceinline__ const typename Epi::Params& epi(int) const { return *ep; }
};

/// Per-instance data of a batched launch (global memory, 64-byte aligned for the descriptors).
template <class Cfg, class RHS, class Epi> struct alignas(64) StageEntry {
    CUtensorMap tmap;
    CentreMaps cmaps;
    StageParams<typename Cfg::T> sp; // ntx, nty, ty, zchunk unused
    RHS rhs;
    typename Epi::Params ep;
};

/// Work source of a persistent batched launch: CTA b processes items b, b + grid, b + 2 grid, ...
/// of a host-built list (instances of any size, tiles x z ranges, longest first).
template <class Cfg, class RHS, class Epi> struct BatchSource {
    using T = typename Cfg::T;
    static constexpr bool kSingleItem = false;
    using Entry = StageEntry<Cfg, RHS, Epi>;
    const Entry* entries;
    const ItemBox* items;
    int nitems, ty_;
    int* err_;
    __device__ __forceinline__ int ty() const { return ty_; }
    __device__ __forceinline__ int* err() const { return err_; }
    __device__ __forceinline__ int count() const {
        return int(blockIdx.x) < nitems ? (nitems - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;
    }
    __device__ __forceinline__ ItemBox item(int m) const { return items[blockIdx.x + size_t(m) * gridDim.x]; }
    __device__ __forceinline__ const CUtensorMap* stencil_map(int i) const { return &entries[i].tmap; }
    __device__ __forceinline__ const CentreMaps& centre_maps(int i) const { return entries[i].cmaps; }
    __device__ __forceinline__ const StageParams<T>& params(int i) const { return entries[i].sp; }
    __device__ __forceinline__ const RHS& rhs_of(int i) const { return entries[i].rhs; }
    __device__ __forceinline__ const typename Epi::Params& epi(int i) const { return entries[i].ep; }
};

/// The stage pipeline of one CTA over the items of a work source. The two rings run on across
/// items: the producer streams the planes of item after item and the consumer warps follow in
/// the same order, so an item's first planes are copied while the previous item's last
/// planes are computed.
template <class Cfg, class RHS, class Epi, class Src> __device__ __forceinline__ void stage_body(const Src& src) {
    using T = typename Cfg::T;
    using RingT = Ring<Cfg, Epi>;
    using C0 = typename RingT::C0;
    using C1 = typename RingT::C1;
    constexpr int G = Cfg::G, NC = Cfg::NC, TX = Cfg::TX, BX = Cfg::BX, XH = Cfg::XH, ZH = Cfg::ZH;
    constexpr int R = RingT::R, RC = RingT::RC, SSLOT = RingT::SSLOT, CSLOT = RingT::CSLOT, NCEN = RingT::NCEN;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* cring = smem_raw + RingT::CRING_OFF;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + RingT::BAR_OFF);
    uint64_t* empty = full + R;
    uint64_t* cempty = empty + R;

    constexpr int CY = Cfg::CY;
    const int TY = src.ty();      // consumer warps
    const int BY = TY * CY + 2 * G;
    const int PNS = BY * BX;      // component stride of the stencil plane inside a slot
    const int CPS = TY * CY * TX; // component stride of a centre-operand box
    const int nitems = src.count();
    if (nitems == 0) return;
    int* const err = src.err();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < R; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], uint32_t(TY));
        }
        for (int s = 0; s < RC; ++s) ptx::mbar_init(&cempty[s], uint32_t(TY));
        ptx::fence_mbar_init();
    }
    __syncthreads();

    if (warp == TY) {
        // ---------------------------------------------------------------- producer warp
        if (lane == 0) {
            const uint32_t bytes = uint32_t(NC * BY * BX * int(sizeof(T)));
            uint32_t cbytes = 0;
            if constexpr (NCEN > 0) cbytes += uint32_t(CPS * NC * int(sizeof(C0)));
            if constexpr (NCEN > 1) cbytes += uint32_t(CPS * NC * int(sizeof(C1)));
            // Plane t (counted over all items) goes to stencil slot ps.s once plane t - R is
            // released (completion t / R of empty[ps.s], parity ps.ph ^ 1). From an item's plane
            // q = 2G on, the same transaction carries the centre operands of its centre plane
            // q - G (z = z0 - 2G + q) into centre slot pc.s, once the centre RC earlier is released.
            RingPos ps, pc;
            long long t = 0, tc = 0;
            bool ok = true;
            unsigned long long wl = kWaitLimitNs;
            for (int m = 0; m < nitems && ok; ++m) {
                const ItemBox b = src.item(m);
                const int skip = src.params(b.inst).skip_plane;
                const int xs = src.params(b.inst).L.xoff - XH; // storage x of the box start minus x0
                wl = src.params(b.inst).wait_ns;
                const CUtensorMap* tmap = src.stencil_map(b.inst);
                const CentreMaps& cm = src.centre_maps(b.inst);
                ptx::prefetch_tensor_map(tmap);
                if constexpr (NCEN > 0) ptx::prefetch_tensor_map(&cm.map[0]);
                if constexpr (NCEN > 1) ptx::prefetch_tensor_map(&cm.map[1]);
                int cx[2] = {0, 0}, cy[2] = {0, 0}, cz[2] = {0, 0};
#pragma unroll
                for (int k = 0; k < NCEN; ++k) {
                    cx[k] = cm.x[k];
                    cy[k] = cm.y[k];
                    cz[k] = cm.z[k];
                }
                const int NP = (b.z1 - b.z0) + 2 * ZH; // planes z0 - ZH .. z1 - 1 + ZH
                for (int q = 0; q < NP; ++q, ++t) {
                    if (t >= R && !ptx::mbar_wait(&empty[ps.s], ps.ph ^ 1u, err, wl)) {
                        ok = false;
                        break;
                    }
                    const bool centre = NCEN > 0 && q >= 2 * ZH;
                    if (centre && tc >= RC && !ptx::mbar_wait(&cempty[pc.s], pc.ph ^ 1u, err, wl)) {
                        ok = false;
                        break;
                    }
                    if (q == skip) {
                        // injected fault: this plane's copy is never issued, so its `full`
                        // barrier never completes and the consumers' bounded waits expire
                        if constexpr (NCEN > 0) {
                            if (centre) {
                                pc.next(RC);
                                ++tc;
                            }
                        }
                        ps.next(R);
                        continue;
                    }
                    ptx::mbar_arrive_expect_tx(&full[ps.s], bytes + (centre ? cbytes : 0u));
                    // storage coordinates: x = x0 - XH + xoff, y = y0 - G + g (= y0), z = z0 - G + q + g;
                    // xoff - XH is 0 or 16 bytes (xoff: ngrow rounded up to 32 bytes, XH: to 16)
                    ptx::tma_load_4d(smem_raw + ps.s * SSLOT, tmap, b.x0 + xs, b.y0, b.z0 + q + (G - ZH), 0,
                                     &full[ps.s]);
                    if constexpr (NCEN > 0) {
                        if (centre) {
                            const int zc = b.z0 - 2 * ZH + q;
                            unsigned char* cs = cring + pc.s * CSLOT;
                            ptx::tma_load_4d(cs + RingT::C0_OFF, &cm.map[0], b.x0 + cx[0], b.y0 + cy[0], zc + cz[0], 0,
                                             &full[ps.s]);
                            if constexpr (NCEN > 1)
                                ptx::tma_load_4d(cs + RingT::C1_OFF, &cm.map[1], b.x0 + cx[1], b.y0 + cy[1],
                                                 zc + cz[1], 0, &full[ps.s]);
                            pc.next(RC);
                            ++tc;
                        }
                    }
                    ps.next(R);
                }
            }
            if (!ok) {
                // a consumer warp stopped releasing slots: let the copies in flight land
                // (bounded: a plane whose copy was never issued completes nothing)
                for (long long r = (t > R ? t - R : 0); r < t; ++r)
                    ptx::mbar_wait(&full[r % R], uint32_t((r / R) & 1), nullptr, wl < 100000000ull ? wl : 100000000ull);
            }
        }
        return;
    }
    if (warp > TY) return;

    // -------------------------------------------------------------------- consumer warps
    constexpr int CX = Cfg::CX, U = Cfg::U;
    constexpr int QL = 2 * ZH + U; // register queue depth (planes)
    // compile-time ring slots: static layout and one item per CTA (the rings start at slot 0)
    constexpr bool kStaticPos = RingT::kStatic && Src::kSingleItem;
    constexpr bool kStaticCen = RingT::kStaticCentre && Src::kSingleItem;
    const bool leader = lane == 0; // the lane that releases ring slots for its warp
    constexpr int NCOL = CY * CX;  // columns (cells per plane) of a thread: column r CX + e is cell (i0 + e, j0 + r)
    const int tx = lane, ty = warp;
    const int coff = (CY * ty + G) * BX + (CX * tx + XH); // cell (i0, j0)'s centre inside the stencil plane (row r: + r BX)
    const int cc = CY * ty * TX + CX * tx;                // ... inside a centre-operand box (row r: + r TX)

    RingPos pos;  // stencil slot of the item's plane it
    RingPos kpos; // centre slot of the item's centre plane it - G
    bool ok = true;
    for (int m = 0; m < nitems && ok; ++m) {
        const ItemBox b = src.item(m);
        // Register copies of everything the plane loop reads: values in kernel-parameter or
        // global space are not known to be loop-invariant, which would keep e.g. the
        // stencils' 1/dx factors and the functor's data inside the loop.
        const RHS f = src.rhs_of(b.inst);
        const StageParams<T>& spr = src.params(b.inst);
        const amrex::GeometryData geom = spr.geom;
        const Layout L = spr.L;
        const double time = spr.time;
        const T* const in = spr.in;
        const unsigned long long wl = spr.wait_ns;
        const int zo = spr.zoff; // the functor sees global z
        const typename Epi::Params epl = src.epi(b.inst);

        const int NP = (b.z1 - b.z0) + 2 * ZH;
        const int i0 = b.x0 + CX * tx, j0 = b.y0 + CY * ty; // this thread's cells: (i0 + e, j0 + r)
        bool act[CY][CX];
#pragma unroll
        for (int r = 0; r < CY; ++r)
#pragma unroll
            for (int e = 0; e < CX; ++e) act[r][e] = (i0 + e < L.n[0]) && (j0 + r < L.n[1]);

        // q[w][m * NC + c]: column w, plane it - 2G - U + m (before the shift of iteration it)
        T q[NCOL][QL * NC];
#pragma unroll
        for (int w = 0; w < NCOL; ++w)
#pragma unroll
            for (int mm = 0; mm < QL * NC; ++mm) q[w][mm] = T(0);

        const T* in_col = in + L.index(i0, j0, 0, 0); // global fallback: cell (i0, j0)'s column at z = 0
        const long long plane = L.px * L.py;

        // Prologue: planes 0 .. 2G-1 (the lower halo and the first G centre planes) into the
        // queue. Planes that are never centre planes (p < G, p >= NP - G) are released once
        // read; every other plane after its iteration as a centre plane.
        RingPos cpos; // stencil slot of plane it - ZH
        if constexpr (ZH == 0) cpos = pos; // the newest plane is the centre plane
#pragma unroll
        for (int p = 0; p < 2 * ZH; ++p) {
            if (p == ZH) cpos = pos;
            // static layout: plane p of the only item sits in slot p (p < 2G < R), first phase
            const int ps = kStaticPos ? p : pos.s;
            const uint32_t pph = kStaticPos ? 0u : pos.ph;
            if (ok && !ptx::mbar_wait(&full[ps], pph, err, wl)) ok = false;
            if (ok) {
                const T* pl = reinterpret_cast<const T*>(smem_raw + ps * SSLOT) + coff;
#pragma unroll
                for (int r = 0; r < CY; ++r)
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        T v[CX];
                        lds<CX>(pl + r * BX + c * PNS, v);
#pragma unroll
                        for (int e = 0; e < CX; ++e) q[r * CX + e][(Cfg::ROT ? p : p + U) * NC + c] = v[e];
                    }
                if (p < ZH || p >= NP - ZH) {
                    __syncwarp();
                    ptx::mbar_arrive_if(&empty[ps], leader);
                }
            }
            if constexpr (!kStaticPos) pos.next(R);
        }
        if (!ok) break;

        // Main loop: U planes per iteration. Cell (e, u) has centre plane it - G + u, i.e.
        // z = z0 - 2G + it + u, and exists while it + u < NP; its queue window is q[e][u ...].
        // Circular queue (ROT): plane p lives in slot p % QL, the loop is unrolled QL times and
        // unrolled copy k (it = 2G + k mod QL) finds offset dk of its centre in slot (G + dk + k) % QL.
        constexpr int KU = Cfg::ROT ? QL : 1;
        uint32_t mph = 0; // static layout: parity of the QL-plane block of this base iteration
        for (int base = 2 * ZH; base < NP && ok; base += KU * U, mph ^= 1u)
#pragma unroll
        for (int k = 0; k < KU; ++k) {
            const int it = base + k * U;
            if (Cfg::ROT && it >= NP) break;
            int su[U], scu[U], sku[U];
            if constexpr (kStaticPos) {
                // it = 2G + QL m + k with R = QL: newest plane in slot (2G + k) % R, in its
                // (m + (2G + k) / R)-th use; centre plane it - G in slot (G + k) % R; centre
                // operands (it - 2G = QL m + k) in slot k % RC when RC divides QL
                su[0] = (2 * ZH + k) % R;
                scu[0] = (ZH + k) % R;
                sku[0] = NCEN == 0 ? 0 : (kStaticCen ? k % RC : kpos.s);
                if (!ptx::mbar_wait(&full[su[0]], mph ^ uint32_t(((2 * ZH + k) / R) & 1), err, wl)) ok = false;
            } else {
                RingPos pp = pos, cp = cpos, kp = kpos;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    su[u] = pp.s;
                    scu[u] = cp.s;
                    sku[u] = kp.s;
                    if (it + u < NP && !ptx::mbar_wait(&full[pp.s], pp.ph, err, wl)) ok = false;
                    pp.next(R);
                    cp.next(R);
                    if constexpr (NCEN > 0) kp.next(RC);
                }
            }
            if (!ok) break;
            if constexpr (!Cfg::ROT) {
#pragma unroll
                for (int w = 0; w < NCOL; ++w)
#pragma unroll
                    for (int mm = 0; mm < 2 * ZH * NC; ++mm) q[w][mm] = q[w][mm + U * NC];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (Cfg::ZQ && (U == 1 || it + u < NP)) {
                    const T* pl = reinterpret_cast<const T*>(smem_raw + su[u] * SSLOT) + coff;
                    const int qs = Cfg::ROT ? (k + 2 * ZH) % QL : 2 * ZH + u; // queue slot of the newest plane
#pragma unroll
                    for (int r = 0; r < CY; ++r)
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            T v[CX];
                            lds<CX>(pl + r * BX + c * PNS, v);
#pragma unroll
                            for (int e = 0; e < CX; ++e) q[r * CX + e][qs * NC + c] = v[e];
                        }
                }
            }

            // all cells' stage values first, then the epilogues (their global stores would
            // otherwise stand between the shared-memory taps of neighbouring cells)
            T kv[U][CY][CX][NC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int z = b.z0 - 2 * ZH + it + u;
                const T* ctr = reinterpret_cast<const T*>(smem_raw + scu[u] * SSLOT) + coff;
#pragma unroll
                for (int r = 0; r < CY; ++r) {
                    // Two cells per thread: the centre row's x taps of both cells (offsets -GW ..
                    // GW + 1 from cell 0, GW = G rounded up to even, GW <= XH) come from registers
                    // filled with aligned vector loads; per-tap loads would be half misaligned
                    // pairs, split into stride-2 scalar loads with two-way bank conflicts.
                    constexpr int GW = (G + 1) / 2 * 2;
                    constexpr int XWN = CX == 2 ? 2 * GW + 2 : 1;
                    static_assert(CX == 1 || GW <= XH, "x window beyond the shared-memory halo");
                    T xwin[NC][XWN];
                    if constexpr (CX == 2) {
#pragma unroll
                        for (int c = 0; c < NC; ++c)
#pragma unroll
                            for (int h = 0; h < XWN / 2; ++h) {
                                T v[2];
                                lds<2>(ctr + r * BX + c * PNS - GW + 2 * h, v);
                                xwin[c][2 * h] = v[0];
                                xwin[c][2 * h + 1] = v[1];
                            }
                    }
                    amrex::StencilView<T> view[CX];
#pragma unroll
                    for (int e = 0; e < CX; ++e)
                        view[e] = amrex::StencilView<T>{ctr + r * BX + e,
                                                        q[r * CX + e] + (Cfg::ROT ? 0 : u * NC),
                                                        in_col + r * L.px + e + z * plane,
                                                        L.px,
                                                        plane,
                                                        L.comp_stride(),
                                                        i0 + e,
                                                        j0 + r,
                                                        z + zo,
                                                        BX,
                                                        PNS,
                                                        ZH,
                                                        Cfg::ZQ ? NC : 0,
                                                        Cfg::ROT ? k : 0,
                                                        Cfg::ROT ? QL : 0,
                                                        CX == 2 ? &xwin[0][0] : nullptr,
                                                        XWN,
                                                        GW + e};
#ifdef TREESAP_B200_CHECK
#pragma unroll
                    for (int e = 0; e < CX; ++e) {
                        // bounds of the stencil slot and of the input field around this cell
                        const int pofs = coff + r * BX + e;
                        const long long gofs = L.index(i0 + e, j0 + r, z, 0);
                        view[e].err = err;
                        view[e].plo = -pofs;
                        view[e].phi = NC * PNS - pofs;
                        view[e].glo = -gofs;
                        view[e].ghi = L.elements() - gofs;
                    }
#endif
                    bool whole = U == 1 || it + u < NP;
#pragma unroll
                    for (int e = 0; e < CX; ++e) whole = whole && act[r][e];
                    if (CX > 1 && whole) {
                        // every cell of the row exists: no per-cell branch, so the taps of
                        // neighbouring cells can share vector loads
#pragma unroll
                        for (int e = 0; e < CX; ++e)
                            eval_cell(f, kv[u][r][e], view[e], in, L, amrex::IntVect{i0 + e, j0 + r, z + zo}, time,
                                      geom, zo);
                    } else {
#pragma unroll
                        for (int e = 0; e < CX; ++e) {
#pragma unroll
                            for (int c = 0; c < NC; ++c) kv[u][r][e][c] = T(0);
                            if ((U == 1 || it + u < NP) && act[r][e])
                                eval_cell(f, kv[u][r][e], view[e], in, L, amrex::IntVect{i0 + e, j0 + r, z + zo}, time,
                                          geom, zo);
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (U == 1 || it + u < NP) {
                    const int z = b.z0 - 2 * ZH + it + u;
                    const unsigned char* cslot = cring + sku[u] * CSLOT;
#pragma unroll
                    for (int r = 0; r < CY; ++r) {
                        const CentreOps<C0, C1> co{reinterpret_cast<const C0*>(cslot + RingT::C0_OFF) + cc + r * TX,
                                                   reinterpret_cast<const C1*>(cslot + RingT::C1_OFF) + cc + r * TX,
                                                   CPS};
                        Epi::template apply<T, NC, CX>(
                            epl, kv[u][r], act[r],
                            reinterpret_cast<const T*>(smem_raw + scu[u] * SSLOT) + coff + r * BX, PNS, i0, j0 + r, z,
                            co);
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (U == 1 || it + u < NP) {
                    ptx::mbar_arrive_if(&empty[scu[u]], leader);
                    if constexpr (NCEN > 0) ptx::mbar_arrive_if(&cempty[sku[u]], leader);
                    if (ZH > 0 && it + u >= NP - ZH) ptx::mbar_arrive_if(&empty[su[u]], leader);
                }
            if constexpr (!kStaticPos) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (U == 1 || it + u < NP) {
                        pos.next(R);
                        cpos.next(R);
                        if constexpr (NCEN > 0) kpos.next(RC);
                    }
                }
            } else if constexpr (NCEN > 0 && !kStaticCen) {
                kpos.next(RC);
            }
        }
    }
}

template <class Cfg, class RHS, class Epi>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MIN_BLOCKS)
    stage_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CentreMaps cmaps,
                 const __grid_constant__ StageParams<typename Cfg::T> sp, const __grid_constant__ RHS rhs,
                 const __grid_constant__ typename Epi::Params ep) {
    const SingleSource<Cfg, RHS, Epi> src{&tmap, &cmaps, &sp, &rhs, &ep};
    stage_body<Cfg, RHS, Epi>(src);
}

/// Persistent batched form: one launch for all items of all instances.
template <class Cfg, class RHS, class Epi>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MIN_BLOCKS)
    batch_stage_kernel(const StageEntry<Cfg, RHS, Epi>* __restrict__ entries, const ItemBox* __restrict__ items,
                       int nitems, int ty, int* err) {
    const BatchSource<Cfg, RHS, Epi> src{entries, items, nitems, ty, err};
    stage_body<Cfg, RHS, Epi>(src);
}

// ------------------------------------------------------------------ epilogues
// Each policy: struct Params; kCentre (0..2) centre-operand fields of element types C0, C1,
// described on the host by centre_src(params, k); and
//   template <T, NC, CX, CO> static void apply(params, k[CX][NC], act[CX], centre, pns, i0, j, z, co)
// for the CX cells (i0 + e, j, z) of a thread (act[e]: the cell exists), where `centre` points
// at component 0 of cell 0's stencil input in shared memory (cell e at centre + e, component
// stride pns) and co.c0 / co.c1 at component 0 of cell 0's centre operands (component stride
// co.cps). i0 is a multiple of CX, so the CX cells of a row form one aligned vector.

/// Epilogue without centre operands.
struct NoCentre {
    static constexpr int kCentre = 0;
    using C0 = char;
    using C1 = char;
    static CentreSrc centre_src(...) { return {}; }
};

/// FP64 plain RK4 stage s with the reference's register scheme
/// (integrators/SingleLevelRK4Integrator.hpp:139-155):
///   s = 0:   acc = init + b k,  arg_next = init + a_next k   (the stencil input is init)
///   s = 1,2: acc += b k,        arg_next = init + a_next k
///   s = 3:   acc += b k
/// Centre operands (s > 0): acc (C0) and, for s < 3, init (C1).
template <int STAGE> struct EpiRK4 {
    struct Params {
        double* acc;
        double* arg_next;
        const double* init;
        Layout L;
        double b, a_next;
    };
    static constexpr int kCentre = STAGE == 0 ? 0 : (STAGE < 3 ? 2 : 1);
    using C0 = double;
    using C1 = double;
    static CentreSrc centre_src(const Params& p, int k) {
        return k == 0 ? CentreSrc{p.acc, p.L, TS_F64} : CentreSrc{p.init, p.L, TS_F64};
    }
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T* centre, int pns, int i0, int j, int z, const CO& co) {
        const long long o0 = p.L.index(i0, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double base_acc[CX], base_init[CX], acc[CX], next[CX];
            if constexpr (STAGE == 0) {
                lds<CX>(centre + c * pns, base_acc);
#pragma unroll
                for (int e = 0; e < CX; ++e) base_init[e] = base_acc[e];
            } else {
                lds<CX>(co.c0 + c * co.cps, base_acc);
                if constexpr (STAGE < 3) lds<CX>(co.c1 + c * co.cps, base_init);
            }
#pragma unroll
            for (int e = 0; e < CX; ++e) {
                acc[e] = base_acc[e] + p.b * k[e][c];
                if constexpr (STAGE < 3) next[e] = base_init[e] + p.a_next * k[e][c];
            }
            stcs<CX>(p.acc + o0 + c * cs, acc, act);
            if constexpr (STAGE < 3) stcs<CX>(p.arg_next + o0 + c * cs, next, act);
        }
    }
};

/// Forward Euler (integrators/SingleLevelEulerIntegrator.hpp:77-84): new = old + dt k.
struct EpiEuler : NoCentre {
    struct Params {
        double* out;
        Layout L;
        double dt;
    };
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T* centre, int pns, int i0, int j, int z, const CO&) {
        const long long o0 = p.L.index(i0, j, z, 0), cs = p.L.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            double u[CX], out[CX];
            lds<CX>(centre + c * pns, u);
#pragma unroll
            for (int e = 0; e < CX; ++e) out[e] = u[e] + p.dt * k[e][c];
            stcs<CX>(p.out + o0 + c * cs, out, act);
        }
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
struct EpiF32S0 : NoCentre {
    struct Params {
        double* k0;
        double* up;
        Layout Lu;
        double dt;
    };
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T* centre, int pns, int i0, int j, int z, const CO&) {
        const long long u0 = p.Lu.index(i0, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            T u[CX];
            lds<CX>(centre + c * pns, u);
            double k0[CX], up[CX];
#pragma unroll
            for (int e = 0; e < CX; ++e) {
                k0[e] = double(k[e][c]);
                up[e] = double(u[e]) + p.dt * double(k[e][c]);
            }
            stcs<CX>(p.k0 + u0 + c * us, k0, act);
            stcs<CX>(p.up + u0 + c * us, up, act);
        }
    }
};

/// Stage 1 of the FP32-stage form: d1 = (dt/2) L k0 from the FP64 k0, stored FP32.
struct EpiF32S1 : NoCentre {
    struct Params {
        float* d1;
        Layout Lf;
        double a_dt;
    };
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&lk)[CX][NC], const bool (&act)[CX],
                                                 const T*, int, int i0, int j, int z, const CO&) {
        const long long o0 = p.Lf.index(i0, j, z, 0), cs = p.Lf.comp_stride();
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            float d[CX];
#pragma unroll
            for (int e = 0; e < CX; ++e) d[e] = static_cast<float>(p.a_dt * double(lk[e][c]));
            stcs<CX>(p.d1 + o0 + c * cs, d, act);
        }
    }
};

/// Stages 2 and 3 of the FP32-stage form. Centre operands of stage 3: d1 (C0, FP32) and
/// u_p (C1, FP64).
template <int STAGE> struct EpiF32Lin {
    struct Params {
        float* d_out;      // stages 1, 2: d1, d2
        const float* d1;   // stage 3
        double* u;         // stage 3: u_p in, u_new out (in place)
        Layout Lf, Lu;
        float a_dt;        // dt/2 (stages 1, 2), dt (stage 3)
        double dt;         // stage 3
    };
    static constexpr int kCentre = STAGE == 3 ? 2 : 0;
    using C0 = float;
    using C1 = double;
    static CentreSrc centre_src(const Params& p, int k) {
        return k == 0 ? CentreSrc{p.d1, p.Lf, TS_F32} : CentreSrc{p.u, p.Lu, TS_F64};
    }
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&lk)[CX][NC], const bool (&act)[CX],
                                                 const T* centre, int pns, int i0, int j, int z, const CO& co) {
        const long long o0 = p.Lf.index(i0, j, z, 0), cs = p.Lf.comp_stride();
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                float d[CX];
#pragma unroll
                for (int e = 0; e < CX; ++e) d[e] = p.a_dt * lk[e][c];
                stcs<CX>(p.d_out + o0 + c * cs, d, act);
            }
        } else if constexpr (STAGE == 2) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                float d1[CX], d[CX];
                lds<CX>(centre + c * pns, d1);
#pragma unroll
                for (int e = 0; e < CX; ++e) d[e] = d1[e] + p.a_dt * lk[e][c];
                stcs<CX>(p.d_out + o0 + c * cs, d, act);
            }
        } else {
            const long long u0 = p.Lu.index(i0, j, z, 0), us = p.Lu.comp_stride();
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                float d1[CX], d2[CX];
                double up[CX], un[CX];
                lds<CX>(co.c0 + c * co.cps, d1);
                lds<CX>(centre + c * pns, d2);
                lds<CX>(co.c1 + c * co.cps, up);
#pragma unroll
                for (int e = 0; e < CX; ++e) {
                    const float d3 = 2.0f * d1[e] + p.a_dt * lk[e][c];
                    const double sum = 2.0 * double(d1[e]) + 2.0 * double(d2[e]) + double(d3);
                    un[e] = up[e] + (p.dt / 6.0) * sum;
                }
                stcs<CX>(p.u + u0 + c * us, un, act);
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

/// z-major grid: tiles of TX x ty CY cells, the z extent split into `nchunks` chunks so that the
/// grid fills the resident CTA slots without chunks shorter than 4G planes (each chunk pays a
/// 2G-plane warm-up).
template <class Cfg> LaunchShape make_shape(const Layout& L, int slots, int ty, int nchunks = 0) {
    LaunchShape s;
    s.ty = ty;
    s.ntx = (L.n[0] + Cfg::TX - 1) / Cfg::TX;
    s.nty = (L.n[1] + ty * Cfg::CY - 1) / (ty * Cfg::CY);
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

/// Resident CTAs per SM of the kernel `K` launched with 32 ty + 32 threads and `smem` bytes of
/// dynamic shared memory, cached per device and tile height; the kernel's dynamic shared-memory
/// limit is raised on the device's first query. A lock guards the cache: integrators on several
/// host threads may query it at once.
template <auto K, int TYMAX> int cached_occupancy(int ty, int smem) {
    static std::mutex m;
    static int occ[64][TYMAX + 1] = {};
    static bool attr[64] = {};
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal beyond the occupancy cache");
    if (ty < 1 || ty > TYMAX) ty = TYMAX;
    std::lock_guard<std::mutex> lock(m);
    if (!attr[dev]) {
        cuda_check(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                   "cudaFuncSetAttribute(smem)");
        attr[dev] = true;
    }
    if (occ[dev][ty] == 0) {
        int nb = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, K, 32 * ty + 32, smem),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        occ[dev][ty] = nb > 0 ? nb : 1;
    }
    return occ[dev][ty];
}

/// Tile height for a given width in x: the largest ty <= TYMAX whose tile count fills the SMs
/// most evenly (fraction of busy slot-time in the last wave), ties to the taller tile.
/// `slots(ty)`: resident CTA slots of the whole GPU for tiles of ty rows.
template <class Cfg, class SlotsFn> int choose_ty(const Layout& L, SlotsFn&& slots) {
    int best = Cfg::TYMAX;
    double best_eff = -1.0;
    for (int ty = Cfg::TYMAX; ty >= (Cfg::TYMAX + 1) / 2; --ty) {
        const int sl = slots(ty);
        const LaunchShape s = make_shape<Cfg>(L, sl, ty);
        const double waves = double(s.grid) / sl;
        const double eff = waves / std::ceil(waves) * (double(ty) / Cfg::TYMAX > 0.75 ? 1.0 : 0.95);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = ty;
        }
    }
    return best;
}

template <class Cfg, class RHS, class Epi> struct StageLauncher {
    using RingT = Ring<Cfg, Epi>;
    static auto kernel() { return &stage_kernel<Cfg, RHS, Epi>; }
    /// Resident CTAs per SM for tiles of `ty` rows.
    static int occupancy(int ty) { return cached_occupancy<&stage_kernel<Cfg, RHS, Epi>, Cfg::TYMAX>(ty, RingT::SMEM); }
    /// Launch shape for a layout; `ty` <= 0 picks the tile height, `nchunks` <= 0 the z split.
    /// The z split fills the resident CTA slots of the chosen tile height.
    static LaunchShape shape(const Layout& L, int sm_count, int ty = 0, int nchunks = 0) {
        if (ty <= 0 || ty > Cfg::TYMAX) ty = choose_ty<Cfg>(L, [&](int t) { return occupancy(t) * sm_count; });
        return make_shape<Cfg>(L, occupancy(ty) * sm_count, ty, nchunks);
    }
    /// The TMA box of the stencil input for a launch shape: (TX + 2 XH) x (ty CY + 2G).
    static int box_x() { return Cfg::BX; }
    static int box_y(const LaunchShape& s) { return s.ty * Cfg::CY + 2 * Cfg::G; }
    /// Centre-operand descriptors (box TX x ty CY) from `map(base, layout, dtype, box_x, box_y)`,
    /// which returns a const CUtensorMap&.
    template <class MapFn>
    static CentreMaps centre_maps(MapFn&& map, const typename Epi::Params& ep, const LaunchShape& s) {
        CentreMaps cm{};
        for (int k = 0; k < Epi::kCentre; ++k) {
            const CentreSrc src = Epi::centre_src(ep, k);
            cm.map[k] = map(src.base, src.L, src.dtype, Cfg::TX, s.ty * Cfg::CY);
            cm.x[k] = src.L.xoff;
            cm.y[k] = src.L.g;
            cm.z[k] = src.L.g;
        }
        return cm;
    }
    static void launch(const CUtensorMap& tmap, const CentreMaps& cmaps, StageParams<typename Cfg::T> sp,
                       const RHS& rhs, const typename Epi::Params& ep, const LaunchShape& s, cudaStream_t stream) {
        sp.ntx = s.ntx;
        sp.nty = s.nty;
        sp.ty = s.ty;
        sp.zchunk = s.zchunk;
        const int threads = 32 * s.ty + 32;
        // Launched through the registered entry point rather than <<< >>>: for some
        // instantiations (template arguments spelled through class-member aliases) the
        // front end's generated launch wrapper resolved to its unspecialised fallback, which
        // launches nothing and reports cudaErrorInvalidDeviceFunction.
        void* args[] = {const_cast<CUtensorMap*>(&tmap), const_cast<CentreMaps*>(&cmaps), &sp,
                        const_cast<RHS*>(&rhs), const_cast<typename Epi::Params*>(&ep)};
        const cudaError_t err = cudaLaunchKernel(reinterpret_cast<const void*>(kernel()), dim3(s.grid), dim3(threads),
                                                 args, size_t(RingT::SMEM), stream);
        if (err != cudaSuccess)
            throw std::runtime_error(std::string("stage_kernel launch (") + __PRETTY_FUNCTION__ +
                                     "): " + cudaGetErrorString(err));
    }
};

} // namespace treesap_b200
