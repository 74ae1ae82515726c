// Host-only AMReX-API shim used by the ORACLE build (test infrastructure, never shipped).
//
// The treesap reference is header-only C++20 on top of AMReX, which is not installed here.
// This file provides the subset of the AMReX API that the reference headers use
// (src/treesap/**, listed in the file's sections below), implemented serially on the host,
// so that the reference's integrator / stencil / decorator / BC headers compile UNCHANGED
// with g++ and can be run as the CPU oracle of the B200 path.
//
// Semantics that live in AMReX rather than in the reference (and that this shim therefore
// restates; parity at this boundary is pinned only by the analytic tests):
//   * Array4 indexing: p[(i-begin.x) + (j-begin.y)*jstride + (k-begin.z)*kstride + n*nstride].
//   * ParallelFor(box, f): k outer, j, i inner (x fastest); large boxes are split over k
//     across host threads (TSREF_THREADS, default all hardware threads).
//   * FillPatchSingleLevel on one level (SingleLevelIntegrator.hpp:153-163):
//       1. every ghost cell whose periodic image (coordinates wrapped in periodic directions)
//          lies inside the domain receives that valid cell's value (FillBoundary);
//       2. every remaining ghost cell, i.e. a cell outside the domain grown by the ghost
//          width in periodic directions only, is passed to the BC functor
//          (GpuBndryFuncFab -> BCType::operator(), DirichletBC.hpp:43-65).
//   * BoxArray::maxSize splits the domain into near-equal boxes of at most block_size.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <type_traits>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include <cstdlib>
#include <thread>

#define AMREX_SPACEDIM 3
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_FORCE_INLINE inline __attribute__((always_inline))
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
#define AMREX_D_DECL(a, b, c) a, b, c

namespace amrex {

using Real = double;
using Long = long long;

// ---------------------------------------------------------------- small value types
struct Dim3 {
    int x, y, z;
};

struct IntVect {
    int vect[3] = {0, 0, 0};
    constexpr IntVect() = default;
    constexpr IntVect(int i, int j, int k) : vect{i, j, k} {}
    constexpr int& operator[](int d) { return vect[d]; }
    constexpr const int& operator[](int d) const { return vect[d]; }
    constexpr IntVect operator-(const IntVect& o) const { return {vect[0] - o[0], vect[1] - o[1], vect[2] - o[2]}; }
    constexpr IntVect operator+(const IntVect& o) const { return {vect[0] + o[0], vect[1] + o[1], vect[2] + o[2]}; }
    constexpr bool operator==(const IntVect& o) const {
        return vect[0] == o[0] && vect[1] == o[1] && vect[2] == o[2];
    }
    const int* getVect() const { return vect; }
};

template <class T, std::size_t N> struct GpuArray {
    T arr[N];
    constexpr T& operator[](int i) { return arr[i]; }
    constexpr const T& operator[](int i) const { return arr[i]; }
    constexpr T* data() { return arr; }
    constexpr const T* data() const { return arr; }
    static constexpr std::size_t size() { return N; }
};

template <class T, std::size_t N> using Array = std::array<T, N>;

template <class T> class Vector : public std::vector<T> {
  public:
    using std::vector<T>::vector;
};

template <class T> constexpr const T& Clamp(const T& v, const T& lo, const T& hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// ---------------------------------------------------------------- Box (cell-centred)
class Box {
  public:
    Box() = default;
    Box(const IntVect& lo, const IntVect& hi) : lo_(lo), hi_(hi) {}
    const IntVect& smallEnd() const { return lo_; }
    const IntVect& bigEnd() const { return hi_; }
    int smallEnd(int d) const { return lo_[d]; }
    int bigEnd(int d) const { return hi_[d]; }
    int length(int d) const { return hi_[d] - lo_[d] + 1; }
    Long numPts() const { return Long(length(0)) * length(1) * length(2); }
    bool ok() const { return hi_[0] >= lo_[0] && hi_[1] >= lo_[1] && hi_[2] >= lo_[2]; }
    Box& grow(int n) {
        for (int d = 0; d < 3; ++d) {
            lo_[d] -= n;
            hi_[d] += n;
        }
        return *this;
    }
    Box& grow(int d, int n) {
        lo_[d] -= n;
        hi_[d] += n;
        return *this;
    }
    bool contains(const IntVect& p) const {
        for (int d = 0; d < 3; ++d)
            if (p[d] < lo_[d] || p[d] > hi_[d]) return false;
        return true;
    }
    bool contains(int i, int j, int k) const { return contains(IntVect{i, j, k}); }

  private:
    IntVect lo_{0, 0, 0}, hi_{-1, -1, -1};
};

inline Box grow(Box b, int n) { return b.grow(n); }

// ---------------------------------------------------------------- Array4
template <class T> struct Array4 {
    T* AMREX_RESTRICT p = nullptr;
    Long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{1, 1, 1}, end{0, 0, 0};
    int ncomp = 0;

    Array4() = default;
    Array4(T* p_, Dim3 b, Dim3 e, int nc)
        : p(p_), jstride(e.x - b.x), kstride(Long(e.x - b.x) * (e.y - b.y)),
          nstride(Long(e.x - b.x) * (e.y - b.y) * (e.z - b.z)), begin(b), end(e), ncomp(nc) {}
    template <class U, class = std::enable_if_t<std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
    Array4(const Array4<U>& o)
        : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride), begin(o.begin), end(o.end),
          ncomp(o.ncomp) {}

    T& operator()(int i, int j, int k, int n = 0) const {
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
    T& operator()(const IntVect& iv, int n = 0) const { return (*this)(iv[0], iv[1], iv[2], n); }
    bool contains(int i, int j, int k) const {
        return i >= begin.x && i < end.x && j >= begin.y && j < end.y && k >= begin.z && k < end.z;
    }
};

// ---------------------------------------------------------------- geometry
namespace CoordSys {
enum CoordType { undef = -1, cartesian = 0, RZ = 1, SPHERICAL = 2 };
}

class RealBox {
  public:
    RealBox() = default;
    RealBox(const Array<Real, 3>& lo, const Array<Real, 3>& hi) : lo_(lo), hi_(hi) {}
    Real lo(int d) const { return lo_[d]; }
    Real hi(int d) const { return hi_[d]; }

  private:
    Array<Real, 3> lo_{0, 0, 0}, hi_{1, 1, 1};
};

struct GeometryData {
    GpuArray<Real, 3> prob_lo, prob_hi, dx;
    Box domain;
    int is_periodic[3] = {0, 0, 0};
    int coord = 0;
    Real CellSize(int d) const { return dx[d]; }
    const Real* CellSize() const { return dx.data(); }
    Real ProbLo(int d) const { return prob_lo[d]; }
    Real ProbHi(int d) const { return prob_hi[d]; }
    const Box& Domain() const { return domain; }
    int isPeriodic(int d) const { return is_periodic[d]; }
};

class Geometry {
  public:
    Geometry() = default;
    Geometry(const Box& dom, const RealBox* rb = nullptr, int coord = 0, int const* is_per = nullptr) {
        d_.domain = dom;
        d_.coord = coord;
        RealBox r = rb ? *rb : RealBox{};
        for (int d = 0; d < 3; ++d) {
            d_.prob_lo[d] = r.lo(d);
            d_.prob_hi[d] = r.hi(d);
            d_.dx[d] = (r.hi(d) - r.lo(d)) / Real(dom.length(d));
            d_.is_periodic[d] = is_per ? is_per[d] : 0;
        }
    }
    Real CellSize(int d) const { return d_.dx[d]; }
    GpuArray<Real, 3> CellSizeArray() const { return d_.dx; }
    GpuArray<Real, 3> ProbLoArray() const { return d_.prob_lo; }
    GpuArray<Real, 3> ProbHiArray() const { return d_.prob_hi; }
    Real ProbLo(int d) const { return d_.prob_lo[d]; }
    const Box& Domain() const { return d_.domain; }
    bool isPeriodic(int d) const { return d_.is_periodic[d] != 0; }
    GeometryData data() const { return d_; }

  private:
    GeometryData d_;
};

// ---------------------------------------------------------------- boundary records
namespace BCType {
enum mathematicalBndryTypes : int {
    bogus = -666,
    reflect_odd = -1,
    int_dir = 0,
    reflect_even = 1,
    foextrap = 2,
    ext_dir = 3,
    hoextrap = 4
};
}

class BCRec {
  public:
    BCRec() = default;
    BCRec(int lx, int ly, int lz, int hx, int hy, int hz) : lo_{lx, ly, lz}, hi_{hx, hy, hz} {}
    int lo(int d) const { return lo_[d]; }
    int hi(int d) const { return hi_[d]; }

  private:
    int lo_[3] = {0, 0, 0}, hi_[3] = {0, 0, 0};
};

// ---------------------------------------------------------------- box decomposition
class BoxArray {
  public:
    BoxArray() = default;
    explicit BoxArray(const Box& b) : boxes_{b} {}
    // Split every box along each direction into near-equal pieces no longer than chunk[d].
    BoxArray& maxSize(const IntVect& chunk) {
        for (int d = 0; d < 3; ++d) {
            std::vector<Box> out;
            for (const Box& b : boxes_) {
                const int len = b.length(d);
                const int nblk = (len + chunk[d] - 1) / chunk[d];
                const int base = len / nblk, extra = len % nblk;
                int lo = b.smallEnd(d);
                for (int q = 0; q < nblk; ++q) {
                    const int sz = base + (q < extra ? 1 : 0);
                    IntVect l = b.smallEnd(), h = b.bigEnd();
                    l[d] = lo;
                    h[d] = lo + sz - 1;
                    out.emplace_back(l, h);
                    lo += sz;
                }
            }
            boxes_ = std::move(out);
        }
        return *this;
    }
    int size() const { return int(boxes_.size()); }
    const Box& operator[](int i) const { return boxes_[i]; }

  private:
    std::vector<Box> boxes_;
};

class DistributionMapping {
  public:
    DistributionMapping() = default;
    explicit DistributionMapping(const BoxArray& ba) : n_(ba.size()) {}

  private:
    int n_ = 0;
};

// ---------------------------------------------------------------- MultiFab
class MFIter;

class MultiFab {
  public:
    MultiFab() = default;
    MultiFab(const BoxArray& ba, const DistributionMapping&, int ncomp, int ngrow)
        : ba_(ba), ncomp_(ncomp), ngrow_(ngrow) {
        data_.resize(ba_.size());
        for (int b = 0; b < ba_.size(); ++b) {
            Box g = ba_[b];
            g.grow(ngrow_);
            data_[b].assign(std::size_t(g.numPts()) * ncomp_, 0.0); // zero-initialised ghosts
        }
    }
    MultiFab(MultiFab&&) noexcept = default;
    MultiFab& operator=(MultiFab&&) noexcept = default;
    MultiFab(const MultiFab&) = delete;
    MultiFab& operator=(const MultiFab&) = delete;

    int nComp() const { return ncomp_; }
    int nGrow() const { return ngrow_; }
    const BoxArray& boxArray() const { return ba_; }
    int size() const { return ba_.size(); }

    Array4<Real> array(int b) {
        Box g = ba_[b];
        g.grow(ngrow_);
        return Array4<Real>(data_[b].data(), Dim3{g.smallEnd(0), g.smallEnd(1), g.smallEnd(2)},
                            Dim3{g.bigEnd(0) + 1, g.bigEnd(1) + 1, g.bigEnd(2) + 1}, ncomp_);
    }
    Array4<const Real> const_array(int b) const { return const_cast<MultiFab*>(this)->array(b); }
    inline Array4<Real> array(const MFIter& mfi);
    inline Array4<const Real> const_array(const MFIter& mfi) const;
    inline Array4<const Real> array(const MFIter& mfi) const;

  private:
    BoxArray ba_;
    int ncomp_ = 0, ngrow_ = 0;
    std::vector<std::vector<Real>> data_;
};

class MFIter {
  public:
    explicit MFIter(const MultiFab& mf) : mf_(&mf) {}
    bool isValid() const { return idx_ < mf_->size(); }
    MFIter& operator++() {
        ++idx_;
        return *this;
    }
    int index() const { return idx_; }
    Box validbox() const { return mf_->boxArray()[idx_]; }
    Box tilebox() const { return validbox(); }

  private:
    const MultiFab* mf_;
    int idx_ = 0;
};

inline Array4<Real> MultiFab::array(const MFIter& mfi) { return array(mfi.index()); }
inline Array4<const Real> MultiFab::const_array(const MFIter& mfi) const { return const_array(mfi.index()); }
inline Array4<const Real> MultiFab::array(const MFIter& mfi) const { return const_array(mfi.index()); }

// ---------------------------------------------------------------- loops
inline int host_threads() {
    static const int n = [] {
        const char* e = std::getenv("TSREF_THREADS");
        int v = e ? std::atoi(e) : int(std::thread::hardware_concurrency());
        return v > 0 ? v : 1;
    }();
    return n;
}

template <class F> void ParallelFor(const Box& bx, F&& f) {
    const int klo = bx.smallEnd(2), khi = bx.bigEnd(2);
    auto slab = [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k)
            for (int j = bx.smallEnd(1); j <= bx.bigEnd(1); ++j)
                for (int i = bx.smallEnd(0); i <= bx.bigEnd(0); ++i)
                    f(i, j, k);
    };
    const int nk = khi - klo + 1;
    const int nt = std::min(host_threads(), nk);
    if (nt <= 1 || bx.numPts() < (Long(1) << 15)) {
        slab(klo, khi + 1);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) {
        const int k0 = klo + int(Long(nk) * t / nt), k1 = klo + int(Long(nk) * (t + 1) / nt);
        pool.emplace_back(slab, k0, k1);
    }
    for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------- ghost fill
template <class F> class GpuBndryFuncFab {
  public:
    explicit GpuBndryFuncFab(const F& f) : f_(f) {}
    const F& user() const { return f_; }

  private:
    F f_;
};

template <class BndryFunc> class PhysBCFunct {
  public:
    PhysBCFunct(const Geometry& geom, const Vector<BCRec>& bcr, const BndryFunc& f)
        : geom_(geom), bcr_(bcr), f_(f) {}

    // Calls the user functor on every ghost cell outside the domain grown (by the ghost
    // width) in the periodic directions only.
    void operator()(MultiFab& mf, int dcomp, int ncomp, const IntVect& nghost, Real time, int bccomp) const {
        const Box& dom = geom_.Domain();
        Box gdom = dom;
        for (int d = 0; d < 3; ++d)
            if (geom_.isPeriodic(d)) gdom.grow(d, nghost[d]);
        const GeometryData gd = geom_.data();
        for (int b = 0; b < mf.size(); ++b) {
            Box g = mf.boxArray()[b];
            g.grow(nghost[0]);
            Array4<Real> a = mf.array(b);
            for (int k = g.smallEnd(2); k <= g.bigEnd(2); ++k)
                for (int j = g.smallEnd(1); j <= g.bigEnd(1); ++j)
                    for (int i = g.smallEnd(0); i <= g.bigEnd(0); ++i) {
                        IntVect iv{i, j, k};
                        if (gdom.contains(iv)) continue;
                        f_.user()(iv, a, dcomp, ncomp, gd, time, bcr_.data() + bccomp, 0, dcomp);
                    }
        }
    }

  private:
    Geometry geom_;
    Vector<BCRec> bcr_;
    BndryFunc f_;
};

// Single-level FillPatch: source == destination in every use by treesap, so only the
// ghost cells are filled (periodic images / other boxes first, then the physical BC).
template <class BC>
void FillPatchSingleLevel(MultiFab& mf, Real time, const Vector<MultiFab*>& smf, const Vector<Real>& /*stime*/,
                          int /*scomp*/, int dcomp, int ncomp, const Geometry& geom, BC& physbcf, int bcfcomp) {
    if (smf.size() != 1 || smf[0] != &mf) {
        std::fprintf(stderr, "oracle shim: FillPatchSingleLevel supports src == dst only\n");
        std::abort();
    }
    const int ng = mf.nGrow();
    const Box& dom = geom.Domain();
    for (int b = 0; b < mf.size(); ++b) {
        Box g = mf.boxArray()[b];
        const Box valid = g;
        g.grow(ng);
        Array4<Real> dst = mf.array(b);
        for (int k = g.smallEnd(2); k <= g.bigEnd(2); ++k)
            for (int j = g.smallEnd(1); j <= g.bigEnd(1); ++j)
                for (int i = g.smallEnd(0); i <= g.bigEnd(0); ++i) {
                    if (valid.contains(i, j, k)) continue;
                    IntVect src{i, j, k};
                    for (int d = 0; d < 3; ++d) {
                        if (!geom.isPeriodic(d)) continue;
                        const int lo = dom.smallEnd(d), len = dom.length(d);
                        src[d] = lo + (((src[d] - lo) % len) + len) % len;
                    }
                    if (!dom.contains(src)) continue; // left for the physical BC
                    for (int s = 0; s < mf.size(); ++s) {
                        if (!mf.boxArray()[s].contains(src)) continue;
                        Array4<const Real> from = mf.const_array(s);
                        for (int n = dcomp; n < dcomp + ncomp; ++n) dst(i, j, k, n) = from(src, n);
                        break;
                    }
                }
    }
    physbcf(mf, dcomp, ncomp, IntVect{ng, ng, ng}, time, bcfcomp);
}

// ---------------------------------------------------------------- misc runtime
inline void Initialize(int&, char**&) {}
inline void Finalize() {}

struct AllPrintStream {
    template <class T> AllPrintStream& operator<<(const T& v) {
        std::cout << v;
        return *this;
    }
    AllPrintStream& operator<<(std::ostream& (*m)(std::ostream&)) {
        m(std::cout);
        return *this;
    }
};
inline AllPrintStream AllPrint() { return {}; }
inline AllPrintStream Print() { return {}; }

inline std::string Concatenate(const std::string& root, int num, int mindigits = 5) {
    std::ostringstream os;
    os << root;
    std::string s = std::to_string(num);
    for (int q = int(s.size()); q < mindigits; ++q) os << '0';
    os << s;
    return os.str();
}

// The oracle writes no plotfiles. The reference calls this only from PlotExporter
// (util/PlotExporter.hpp:54-59), at the start of pre_step(), with the integrator's
// state_old; the oracle driver installs a hook here to read and seed that state through
// the reference's own public configureExporter() API.
using PlotHook = void (*)(void* user, const MultiFab& mf, int step, Real time);
inline PlotHook& plot_hook() {
    static PlotHook h = nullptr;
    return h;
}
inline void*& plot_hook_user() {
    static void* u = nullptr;
    return u;
}
inline void WriteSingleLevelPlotfile(const std::string&, const MultiFab& mf, const Vector<std::string>&,
                                     const Geometry&, Real time, int step) {
    if (plot_hook()) plot_hook()(plot_hook_user(), mf, step, time);
}

} // namespace amrex
