// treesap-b200 engine: HBM layout of a field and an owning device buffer.
//
// Layout (see include/treesap_b200.h): [comp][z][y][x], x fastest, ngrow ghost cells on every
// face, x origin shifted by xoff = ngrow rounded up to 16 bytes so interior rows start 16-byte
// aligned (and TMA boxes that start ngrow cells left of a tile start on a 16-byte boundary),
// row pitch padded to 16 bytes (TMA stride rule).
#pragma once

#include <AMReX.H>
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include <treesap_b200.h>

namespace treesap_b200 {

struct Layout {
    int n[3] = {0, 0, 0};
    int g = 0;
    int nc = 0;
    int esize = 8;
    int xoff = 0;
    long long px = 0, py = 0, pz = 0;

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE long long comp_stride() const { return px * py * pz; }
    /// Row (k, j) of a component as a 32-bit number (make() guarantees py pz < 2^31), widened once
    /// by the row pitch: one 32x32->64 multiply per index instead of 64-bit products.
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE long long index(int i, int j, int k, int c) const {
        const int row = (k + g) * int(py) + (j + g);
        return c * comp_stride() + (long long)row * int(px) + (i + xoff);
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE long long elements() const { return comp_stride() * nc; }
    long long bytes() const { return elements() * esize; }
    long long valid_cells() const { return (long long)n[0] * n[1] * n[2]; }

    static int round_up(int v, int m) { return (v + m - 1) / m * m; }
    static Layout make(const int n_[3], int g_, int nc_, int esize_) {
        Layout L;
        for (int d = 0; d < 3; ++d) L.n[d] = n_[d];
        L.g = g_;
        L.nc = nc_;
        L.esize = esize_;
        // x origin and row pitch on 32-byte sector boundaries: rows of valid cells then start and
        // end on whole sectors wherever the extent allows, so stores of whole rows leave no
        // partly written sector for the memory to read back
        const int a = 32 / esize_;
        L.xoff = round_up(g_, a);
        L.px = round_up(L.xoff + n_[0] + g_, a);
        L.py = n_[1] + 2 * g_;
        L.pz = n_[2] + 2 * g_;
        if (!rows_fit(n_, g_)) throw std::invalid_argument("field extents beyond 2^31 rows per component");
        return L;
    }
    /// Whether index() can count the rows (y-z) of one component and the row pitch in 32 bits.
    static bool rows_fit(const int n_[3], int g_) {
        const long long py_ = (long long)n_[1] + 2 * g_, pz_ = (long long)n_[2] + 2 * g_;
        const long long px_ = (long long)n_[0] + 4 * g_ + 8;
        return py_ * pz_ < (1LL << 31) && px_ < (1LL << 31);
    }
    ts_field_layout to_c(int dtype) const {
        ts_field_layout c{};
        for (int d = 0; d < 3; ++d) c.n[d] = n[d];
        c.ngrow = g;
        c.ncomp = nc;
        c.dtype = dtype;
        c.xoff = xoff;
        c.px = px;
        c.py = py;
        c.pz = pz;
        return c;
    }
};

/// Plain (view-less) Array4 over a field, with AMReX's index convention. `zoff`: global z index
/// of the field's plane 0 (a z slab of a larger domain), so that the Array4 takes global indices.
template <class T> AMREX_GPU_HOST_DEVICE inline amrex::Array4<T> make_array4(T* base, const Layout& L, int zoff = 0) {
    return amrex::Array4<T>(base, L.px, L.px * L.py, L.comp_stride(), amrex::Dim3{-L.xoff, -L.g, zoff - L.g},
                            amrex::Dim3{int(L.px) - L.xoff, L.n[1] + L.g, zoff + L.n[2] + L.g}, L.nc);
}

/// Where a field sits in a domain decomposed into z slabs: its plane 0 is global plane `zoff`
/// of a domain `nz` planes deep, and its lower / upper ghost planes are filled by a halo
/// exchange with the neighbouring slabs (`lo_ex` / `hi_ex`) rather than by the ghost fill.
/// The default (nz = 0) is a single box: the field is the whole domain.
struct SlabZ {
    int zoff = 0;
    int nz = 0;
    int lo_ex = 0, hi_ex = 0;
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        // clear the runtime's last-error slot (a failed cudaMalloc leaves its error there, and the
        // next launch check would report it again); sticky errors stay reported by every call
        (void)cudaGetLastError();
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

/// Pending injected allocation failures of the calling host thread (ts_context_inject_fault,
/// TS_FAULT_ALLOC): while positive, each DeviceField allocation fails as out of memory
/// without calling cudaMalloc, and decrements it.
inline int& alloc_faults() {
    static thread_local int n = 0;
    return n;
}

/// Owning, zero-initialised device buffer of one field.
template <class T> class DeviceField {
  public:
    DeviceField() = default;
    DeviceField(const int n[3], int g, int nc) : L_(Layout::make(n, g, nc, sizeof(T))) {
        if (alloc_faults() > 0) {
            --alloc_faults();
            throw std::runtime_error("cudaMalloc(field): out of memory (injected)");
        }
        cuda_check(cudaMalloc(&p_, L_.bytes()), "cudaMalloc(field)");
        cuda_check(cudaMemset(p_, 0, L_.bytes()), "cudaMemset(field)");
    }
    DeviceField(DeviceField&& o) noexcept : L_(o.L_), p_(o.p_) { o.p_ = nullptr; }
    DeviceField& operator=(DeviceField&& o) noexcept {
        if (this != &o) {
            release();
            L_ = o.L_;
            p_ = o.p_;
            o.p_ = nullptr;
        }
        return *this;
    }
    DeviceField(const DeviceField&) = delete;
    DeviceField& operator=(const DeviceField&) = delete;
    ~DeviceField() { release(); }

    T* data() const { return p_; }
    const Layout& layout() const { return L_; }
    amrex::Array4<T> array() const { return make_array4(p_, L_); }
    amrex::Array4<const T> const_array() const { return make_array4<const T>(p_, L_); }
    friend void swap(DeviceField& a, DeviceField& b) noexcept {
        std::swap(a.L_, b.L_);
        std::swap(a.p_, b.p_);
    }

  private:
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
    }
    Layout L_{};
    T* p_ = nullptr;
};

} // namespace treesap_b200
