// treesap-b200 engine: ghost fill, initialisation and host-order pack/unpack kernels.
//
// Ghost fill (the single-level FillPatch of SingleLevelIntegrator.hpp:153-163): each thread
// fills a few ghost cells, all components. A ghost cell whose coordinates, wrapped in the periodic
// directions, land inside the domain takes that valid cell's value; every other ghost cell
// (outside the domain grown by the ghost width in periodic directions only) is handed to
// the model's BC functor (DirichletBC.hpp:43-65 writes its values to all components,
// NoOpBC leaves the cell alone). The ghost cells are enumerated slab by slab so that all
// z- and y-face writes are contiguous along x:
//   z slabs: k in [-g,0) u [n2, n2+g), all j, i          (2 g (n1+2g)(n0+2g) cells)
//   y slabs: k in [0,n2), j in [-g,0) u [n1,n1+g), all i (2 g n2 (n0+2g) cells)
//   x slabs: k in [0,n2), j in [0,n1), i in [-g,0) u [n0,n0+g)  (2 g n2 n1 cells)
#pragma once

#include <AMReX.H>
#include <cuda_runtime.h>

#include <type_traits>

#include "../util/static_for.hpp"
#include "field.hpp"

namespace treesap_b200 {

enum class GhostMode : int {
    Functor = 0,     // periodic images + the BC functor outside the domain
    Homogeneous = 1, // periodic images + zero outside the domain (increments of Dirichlet data)
    PeriodicOnly = 2 // periodic images only (ghosts outside the domain untouched)
};

struct GhostCount {
    long long z, y, x;
    AMREX_GPU_HOST_DEVICE long long total() const { return z + y + x; }
};

AMREX_GPU_HOST_DEVICE inline GhostCount ghost_count(const Layout& L) {
    const long long g = L.g, n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    return {2 * g * (n1 + 2 * g) * (n0 + 2 * g), 2 * g * n2 * (n0 + 2 * g), 2 * g * n2 * n1};
}

AMREX_GPU_HOST_DEVICE inline void ghost_coords(const Layout& L, long long t, int& i, int& j, int& k) {
    const GhostCount gc = ghost_count(L);
    const int g = L.g, n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    if (gc.total() < (1LL << 31)) {
        // the same enumeration in 32-bit arithmetic (64-bit divisions cost several times more)
        const unsigned row = unsigned(n0 + 2 * g), twog = unsigned(2 * g);
        unsigned u = unsigned(t);
        if (u < unsigned(gc.z)) {
            const unsigned q = u / row, rows = unsigned(n1 + 2 * g);
            i = int(u - q * row) - g;
            const unsigned kk = q / rows;
            j = int(q - kk * rows) - g;
            k = int(kk) < g ? int(kk) - g : n2 + (int(kk) - g);
            return;
        }
        u -= unsigned(gc.z);
        if (u < unsigned(gc.y)) {
            const unsigned q = u / row;
            i = int(u - q * row) - g;
            const unsigned kq = q / twog;
            const int jj = int(q - kq * twog);
            k = int(kq);
            j = jj < g ? jj - g : n1 + (jj - g);
            return;
        }
        u -= unsigned(gc.y);
        const unsigned q = u / twog;
        const int ii = int(u - q * twog);
        const unsigned kq = q / unsigned(n1);
        k = int(kq);
        j = int(q - kq * unsigned(n1));
        i = ii < g ? ii - g : n0 + (ii - g);
        return;
    }
    if (t < gc.z) {
        const long long row = n0 + 2 * g, plane = row * (n1 + 2 * g);
        const int kk = int(t / plane);
        const long long r = t % plane;
        j = int(r / row) - g;
        i = int(r % row) - g;
        k = kk < g ? kk - g : n2 + (kk - g);
        return;
    }
    t -= gc.z;
    if (t < gc.y) {
        const long long row = n0 + 2 * g, plane = row * 2 * g;
        k = int(t / plane);
        const long long r = t % plane;
        const int jj = int(r / row);
        i = int(r % row) - g;
        j = jj < g ? jj - g : n1 + (jj - g);
        return;
    }
    t -= gc.y;
    const long long plane = (long long)n1 * 2 * g;
    k = int(t / plane);
    const long long r = t % plane;
    j = int(r / (2 * g));
    const int ii = int(r % (2 * g));
    i = ii < g ? ii - g : n0 + (ii - g);
}

/// What the fill does with one ghost cell: its storage offset, and for a periodic image the
/// offset of the valid cell it copies.
struct GhostTarget {
    enum Kind : int { Skip = 0, Copy = 1, Zero = 2, Functor = 3 };
    long long dst, src;
    int kind;
};

/// Resolves ghost cell number t of a field (slab enumeration of ghost_coords).
/// For a z slab (sz.nz > 0) the ghost cells of exchange planes (sz.lo_ex / sz.hi_ex) are left to
/// the halo exchange, and the domain tests and the BC functor use global z (local + sz.zoff);
/// the periodic source of every other ghost cell lies in the slab's own planes, so a source is
/// always a valid cell and never another ghost cell of the same fill.
__device__ __forceinline__ GhostTarget ghost_target(const Layout& L, const amrex::GeometryData& geom, int mode,
                                                    long long t, const SlabZ& sz) {
    int i, j, k;
    ghost_coords(L, t, i, j, k);
    if ((k < 0 && sz.lo_ex) || (k >= L.n[2] && sz.hi_ex)) return {0, 0, GhostTarget::Skip};
    const int nzg = sz.nz > 0 ? sz.nz : L.n[2];
    const int n[3] = {L.n[0], L.n[1], nzg};
    int s[3] = {i, j, k + sz.zoff};
    bool inside = true;
    for (int d = 0; d < 3; ++d) {
        // a ghost coordinate lies within one period of the domain when ngrow <= n, so the
        // periodic image is one conditional shift (an integer modulo by a run-time n costs
        // dozens of instructions, and this runs for every ghost cell of every fill); smaller
        // domains take more shifts
        if (geom.is_periodic[d]) {
            while (s[d] < 0) s[d] += n[d];
            while (s[d] >= n[d]) s[d] -= n[d];
        }
        if (s[d] < 0 || s[d] >= n[d]) inside = false;
    }
    const long long dst = L.index(i, j, k, 0);
    if (inside) return {dst, L.index(s[0], s[1], s[2] - sz.zoff, 0), GhostTarget::Copy};
    if (mode == int(GhostMode::Homogeneous)) return {dst, 0, GhostTarget::Zero};
    if (mode == int(GhostMode::Functor)) return {dst, 0, GhostTarget::Functor};
    return {0, 0, GhostTarget::Skip};
}

/// Fills ghost cells t0, t0 + step, ..., t0 + (K-1) step (those below `end`) of field f.
/// The K cells are resolved first and each component's K source values are loaded before any
/// is stored, so a thread keeps K loads in flight: one load-store pair at a time leaves too
/// few bytes in flight per SM to cover the DRAM latency, and the fill then runs at about
/// half the HBM bandwidth.
template <int K, class T, class BC>
__device__ __forceinline__ void ghost_fill_cells(T* __restrict__ f, const Layout& L, const amrex::GeometryData& geom,
                                                 const BC& bc, const amrex::BCRec* bcr, double time, int mode,
                                                 long long t0, long long step, long long end,
                                                 const SlabZ& sz = SlabZ{}) {
    GhostTarget tg[K];
    unsigned functor_cells = 0;
#pragma unroll
    for (int u = 0; u < K; ++u) {
        const long long t = t0 + u * step;
        tg[u] = t < end ? ghost_target(L, geom, mode, t, sz) : GhostTarget{0, 0, GhostTarget::Skip};
        if (tg[u].kind == GhostTarget::Functor) functor_cells |= 1u << u;
    }
    const long long cs = L.comp_stride();
    for (int c = 0; c < L.nc; ++c) {
        T v[K];
#pragma unroll
        for (int u = 0; u < K; ++u) v[u] = tg[u].kind == GhostTarget::Copy ? f[tg[u].src + c * cs] : T(0);
#pragma unroll
        for (int u = 0; u < K; ++u)
            if (tg[u].kind == GhostTarget::Copy || tg[u].kind == GhostTarget::Zero) f[tg[u].dst + c * cs] = v[u];
    }
    if constexpr (std::is_same_v<T, amrex::Real>) {
        // cells outside the domain (non-periodic faces) go to the model's BC functor one by one
        while (functor_cells) {
            const int u = __ffs(int(functor_cells)) - 1;
            functor_cells &= functor_cells - 1;
            int i, j, k;
            ghost_coords(L, t0 + u * step, i, j, k);
            const amrex::Array4<amrex::Real> dest = make_array4(f, L, sz.zoff);
            bc(amrex::IntVect{i, j, k + sz.zoff}, dest, 0, L.nc, geom, time, bcr, 0, 0);
        }
    }
}

/// Ghost cells per thread and pass of the single-field fill.
constexpr int kGhostUnroll = 4;

template <class T, class BC>
__global__ void ghost_fill_kernel(T* __restrict__ f, const Layout L, const amrex::GeometryData geom, const BC bc,
                                  const amrex::BCRec* bcr, double time, int mode, const SlabZ sz) {
    const long long total = ghost_count(L).total();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += kGhostUnroll * stride)
        ghost_fill_cells<kGhostUnroll>(f, L, geom, bc, bcr, time, mode, t, stride, total, sz);
}

/// One field of a batched ghost fill.
template <class T, class BC> struct GhostEntry {
    T* f;
    Layout L;
    amrex::GeometryData geom;
    BC bc;
    double time;
    int mode;
};

/// A run of `kGhostChunk` consecutive ghost cells (or fewer, at the end) of one entry.
struct GhostChunk {
    int entry;
    int pad;
    long long first;
};
constexpr int kGhostChunk = 2048;

/// Threads of a batched ghost-fill block, and the ghost cells each fills per pass: 3 cells
/// fit the 64 registers of 4 blocks per SM without spills (4 cells spilled into local memory,
/// whose traffic nearly matched the fill's own loads).
constexpr int kGhostFillThreads = 256;
constexpr int kBatchGhostUnroll = 3;

/// Ghost fill of many fields in one launch: block b fills the ghost cells of chunk b (its
/// entry read once per block from global memory into shared memory). At least 4 blocks per SM
/// (64 registers a thread): 1024 threads per SM, each with kBatchGhostUnroll loads in flight.
template <class T, class BC>
__global__ void __launch_bounds__(kGhostFillThreads, 4) batch_ghost_fill_kernel(const GhostEntry<T, BC>* __restrict__ entries,
                                                                            const GhostChunk* __restrict__ chunks,
                                                                            int nchunks, const amrex::BCRec* bcr) {
    using E = GhostEntry<T, BC>;
    constexpr int K = kBatchGhostUnroll;
    __shared__ __align__(16) unsigned char raw[sizeof(E)];
    auto& e = *reinterpret_cast<E*>(raw);
    for (int b = blockIdx.x; b < nchunks; b += gridDim.x) {
        const GhostChunk ch = chunks[b];
        __syncthreads(); // the previous chunk's threads are done with the entry
        if constexpr (std::is_trivially_copyable_v<E> && sizeof(E) % 8 == 0 && alignof(E) >= 8) {
            // one 8-byte word per thread: a single memory round trip instead of thread 0's serial copy
            const auto* q = reinterpret_cast<const unsigned long long*>(entries + ch.entry);
            auto* r = reinterpret_cast<unsigned long long*>(raw);
            for (int w = threadIdx.x; w < int(sizeof(E) / 8); w += blockDim.x) r[w] = q[w];
        } else {
            if (threadIdx.x == 0) e = entries[ch.entry];
        }
        __syncthreads();
        const long long total = ghost_count(e.L).total();
        const long long end = ch.first + kGhostChunk < total ? ch.first + kGhostChunk : total;
        for (long long t = ch.first + threadIdx.x; t < end; t += (long long)K * blockDim.x)
            ghost_fill_cells<K>(e.f, e.L, e.geom, e.bc, bcr, e.time, e.mode, t, blockDim.x, end);
    }
}

template <class T, class BC>
void launch_ghost_fill(T* f, const Layout& L, const amrex::GeometryData& geom, const BC& bc, const amrex::BCRec* bcr,
                       double time, GhostMode mode, int sm_count, cudaStream_t stream, const SlabZ& sz = SlabZ{}) {
    const long long total = ghost_count(L).total();
    if (total == 0) return;
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    const long long cap = (long long)sm_count * 16;
    if (blocks > cap) blocks = cap;
    ghost_fill_kernel<T, BC><<<int(blocks), threads, 0, stream>>>(f, L, geom, bc, bcr, time, int(mode), sz);
    cuda_check(cudaGetLastError(), "ghost_fill_kernel launch");
}

/// Halo exchange between z slabs: copies the valid x-y region of `np` planes, all components,
/// into planes [kd0, kd0 + np) of field `dst` (layout Ld) from a source with the same x-y
/// geometry (px, py, xoff, ghost width): element (i, j, p, c) of the source is at
/// src[c * src_cs + p * px * py + (j + g) * px + i + xoff] (src: a neighbour field from its
/// plane ks0 on, or a staging buffer of whole planes received from another GPU).
template <class T>
__global__ void __launch_bounds__(128) halo_copy_kernel(T* __restrict__ dst, const Layout Ld, int kd0,
                                                        const T* __restrict__ src, long long src_cs, int np) {
    // one row (c, p, j) per block iteration, its cells over the threads: the per-row index split
    // is block-uniform, so no thread divides
    const int rows = Ld.n[1];
    const long long nrows = (long long)Ld.nc * np * rows, plane = Ld.px * Ld.py;
    for (long long q = blockIdx.x; q < nrows; q += gridDim.x) {
        const int j = int(q % rows);
        const long long cp = q / rows;
        const int p = int(cp % np), c = int(cp / np);
        T* d = dst + Ld.index(0, j, kd0 + p, c);
        const T* s = src + c * src_cs + p * plane + (long long)(j + Ld.g) * Ld.px + Ld.xoff;
        for (int i = threadIdx.x; i < Ld.n[0]; i += blockDim.x) d[i] = s[i];
    }
}

template <class T>
void launch_halo_copy(T* dst, const Layout& Ld, int kd0, const T* src, long long src_cs, int np, int sm_count,
                      cudaStream_t stream) {
    const long long nrows = (long long)Ld.nc * np * Ld.n[1];
    if (nrows == 0 || Ld.n[0] == 0) return;
    long long blocks = nrows;
    if (blocks > (long long)sm_count * 32) blocks = (long long)sm_count * 32;
    halo_copy_kernel<T><<<int(blocks), 128, 0, stream>>>(dst, Ld, kd0, src, src_cs, np);
    cuda_check(cudaGetLastError(), "halo_copy_kernel launch");
}

/// initialise(): state(i,j,k,c) = init<c>(lo + (i + 1/2) dx, ...) (SingleLevelIntegrator.hpp:84-92).
/// `zoff`: global z index of the field's plane 0 (z slabs).
template <int NC, class Init>
__global__ void init_kernel(double* __restrict__ f, const Layout L, const amrex::GeometryData geom, const Init init,
                            int zoff = 0) {
    const long long ncell = (long long)L.n[0] * L.n[1] * L.n[2];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = int(t % L.n[0]), j = int((t / L.n[0]) % L.n[1]), k = int(t / ((long long)L.n[0] * L.n[1]));
        const double x = geom.prob_lo[0] + (i + 0.5) * geom.dx[0];
        const double y = geom.prob_lo[1] + (j + 0.5) * geom.dx[1];
        const double z = geom.prob_lo[2] + (k + zoff + 0.5) * geom.dx[2];
        const long long o = L.index(i, j, k, 0), cs = L.comp_stride();
        treesap::static_for<NC>([&]<int c>() { f[o + c * cs] = init.template operator()<c>(x, y, z); });
    }
}

/// Health check: sets *flag to 1 when any valid cell of any component is NaN or infinite.
template <class T> __global__ void nonfinite_kernel(const T* __restrict__ f, const Layout L, int* flag) {
    const long long ncell = (long long)L.n[0] * L.n[1] * L.n[2];
    const long long total = ncell * L.nc;
    bool bad = false;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = int(t / ncell);
        const long long r = t % ncell;
        const int i = int(r % L.n[0]), j = int((r / L.n[0]) % L.n[1]), k = int(r / ((long long)L.n[0] * L.n[1]));
        bad = bad || !isfinite(f[L.index(i, j, k, c)]);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

/// Enqueues the health check of one field; `flag` (device int) must be zero beforehand.
template <class T> void launch_nonfinite(const T* f, const Layout& L, int* flag, int sm_count, cudaStream_t stream) {
    const long long total = L.valid_cells() * L.nc;
    long long blocks = (total + 255) / 256;
    if (blocks > (long long)sm_count * 16) blocks = (long long)sm_count * 16;
    if (blocks < 1) blocks = 1;
    nonfinite_kernel<T><<<int(blocks), 256, 0, stream>>>(f, L, flag);
    cuda_check(cudaGetLastError(), "nonfinite_kernel launch");
}

/// Contiguous valid-cell order [comp][z][y][x] <-> field layout. dir = 0: packed -> field; 1: field -> packed.
template <class T>
__global__ void pack_kernel(T* __restrict__ f, const Layout L, T* __restrict__ packed, int dir) {
    const long long ncell = (long long)L.n[0] * L.n[1] * L.n[2];
    const long long total = ncell * L.nc;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = int(t / ncell);
        const long long r = t % ncell;
        const int i = int(r % L.n[0]), j = int((r / L.n[0]) % L.n[1]), k = int(r / ((long long)L.n[0] * L.n[1]));
        const long long o = L.index(i, j, k, c);
        if (dir == 0)
            f[o] = packed[t];
        else
            packed[t] = f[o];
    }
}

template <class T>
void launch_pack(T* f, const Layout& L, T* packed, int dir, int sm_count, cudaStream_t stream) {
    const long long total = L.valid_cells() * L.nc;
    long long blocks = (total + 255) / 256;
    if (blocks > (long long)sm_count * 32) blocks = (long long)sm_count * 32;
    pack_kernel<T><<<int(blocks), 256, 0, stream>>>(f, L, packed, dir);
    cuda_check(cudaGetLastError(), "pack_kernel launch");
}

} // namespace treesap_b200
