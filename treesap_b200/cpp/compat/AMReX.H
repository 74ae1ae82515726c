// treesap-b200: minimal, device-capable `amrex` compatibility layer.
//
// treesap user models are written against a handful of AMReX types (Real, IntVect, Array4,
// GeometryData, Geometry, Box, RealBox, GpuArray, Array, Vector, BCRec, BCType, Clamp and
// the AMREX_* macros; reference pde-model/PDEModelConcepts.hpp:44-139 and the examples).
// This header provides exactly those, so that models compile unchanged without AMReX.
// Nothing here allocates device memory or launches work: the engine in
// treesap/engine/ owns that.
//
// Array4 extension: an Array4<const T> may carry a pointer to a `StencilView`, which the
// fused stage kernels set up per thread and per cell. With a view, element (i,j,k,n) is
// read from the kernel's shared-memory plane (same z as the stencil centre), from the
// thread's register queue (same x and y as the centre) or, for any other offset, from
// global memory. Inside the engine the view and the centre are known after inlining, so
// every `arr(i+s, j, k, n)` of a user stencil becomes one shared-memory load with an
// immediate offset or one register. Without a view (the default), Array4 indexes its
// pointer exactly like AMReX: p[(i-begin.x) + (j-begin.y)*jstride + (k-begin.z)*kstride + n*nstride].
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#if defined(__CUDACC__)
#define AMREX_GPU_HOST_DEVICE __host__ __device__
#define AMREX_GPU_DEVICE __device__
#define AMREX_GPU_HOST __host__
#define AMREX_FORCE_INLINE __forceinline__
#else
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_FORCE_INLINE inline __attribute__((always_inline))
#endif
#define AMREX_INLINE inline
#define AMREX_RESTRICT __restrict__
#define AMREX_SPACEDIM 3
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_USE_GPU 1
#define AMREX_USE_CUDA 1

namespace amrex {

using Real = double;
using Long = long long;

struct Dim3 {
    int x, y, z;
};

// ------------------------------------------------------------------ IntVect
struct IntVect {
    int vect[3] = {0, 0, 0};
    AMREX_GPU_HOST_DEVICE constexpr IntVect() {}
    AMREX_GPU_HOST_DEVICE constexpr IntVect(int i, int j, int k) : vect{i, j, k} {}
    AMREX_GPU_HOST_DEVICE constexpr int& operator[](int d) { return vect[d]; }
    AMREX_GPU_HOST_DEVICE constexpr const int& operator[](int d) const { return vect[d]; }
    AMREX_GPU_HOST_DEVICE constexpr IntVect operator+(const IntVect& o) const {
        return {vect[0] + o[0], vect[1] + o[1], vect[2] + o[2]};
    }
    AMREX_GPU_HOST_DEVICE constexpr IntVect operator-(const IntVect& o) const {
        return {vect[0] - o[0], vect[1] - o[1], vect[2] - o[2]};
    }
    AMREX_GPU_HOST_DEVICE constexpr bool operator==(const IntVect& o) const {
        return vect[0] == o[0] && vect[1] == o[1] && vect[2] == o[2];
    }
    AMREX_GPU_HOST_DEVICE constexpr bool operator!=(const IntVect& o) const { return !(*this == o); }
    AMREX_GPU_HOST_DEVICE constexpr Dim3 dim3() const { return {vect[0], vect[1], vect[2]}; }
    const int* getVect() const { return vect; }
};

// ------------------------------------------------------------------ containers
template <class T, std::size_t N> struct GpuArray {
    T arr[N];
    AMREX_GPU_HOST_DEVICE constexpr T& operator[](int i) { return arr[i]; }
    AMREX_GPU_HOST_DEVICE constexpr const T& operator[](int i) const { return arr[i]; }
    AMREX_GPU_HOST_DEVICE constexpr T* data() { return arr; }
    AMREX_GPU_HOST_DEVICE constexpr const T* data() const { return arr; }
    AMREX_GPU_HOST_DEVICE static constexpr std::size_t size() { return N; }
};

template <class T, std::size_t N> using Array = std::array<T, N>;

template <class T> class Vector : public std::vector<T> {
  public:
    using std::vector<T>::vector;
};

template <class T>
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr const T& Clamp(const T& v, const T& lo, const T& hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// ------------------------------------------------------------------ Box (cell-centred, inclusive bounds)
class Box {
  public:
    AMREX_GPU_HOST_DEVICE constexpr Box() {}
    AMREX_GPU_HOST_DEVICE constexpr Box(const IntVect& lo, const IntVect& hi) : lo_(lo), hi_(hi) {}
    AMREX_GPU_HOST_DEVICE constexpr const IntVect& smallEnd() const { return lo_; }
    AMREX_GPU_HOST_DEVICE constexpr const IntVect& bigEnd() const { return hi_; }
    AMREX_GPU_HOST_DEVICE constexpr int smallEnd(int d) const { return lo_[d]; }
    AMREX_GPU_HOST_DEVICE constexpr int bigEnd(int d) const { return hi_[d]; }
    AMREX_GPU_HOST_DEVICE constexpr int length(int d) const { return hi_[d] - lo_[d] + 1; }
    AMREX_GPU_HOST_DEVICE constexpr IntVect length() const { return {length(0), length(1), length(2)}; }
    AMREX_GPU_HOST_DEVICE constexpr Long numPts() const {
        return ok() ? Long(length(0)) * length(1) * length(2) : 0;
    }
    AMREX_GPU_HOST_DEVICE constexpr bool ok() const {
        return hi_[0] >= lo_[0] && hi_[1] >= lo_[1] && hi_[2] >= lo_[2];
    }
    AMREX_GPU_HOST_DEVICE constexpr Box& grow(int n) {
        for (int d = 0; d < 3; ++d) {
            lo_[d] -= n;
            hi_[d] += n;
        }
        return *this;
    }
    AMREX_GPU_HOST_DEVICE constexpr Box& grow(int d, int n) {
        lo_[d] -= n;
        hi_[d] += n;
        return *this;
    }
    AMREX_GPU_HOST_DEVICE constexpr bool contains(const IntVect& p) const {
        return p[0] >= lo_[0] && p[0] <= hi_[0] && p[1] >= lo_[1] && p[1] <= hi_[1] && p[2] >= lo_[2] &&
               p[2] <= hi_[2];
    }
    AMREX_GPU_HOST_DEVICE constexpr bool contains(int i, int j, int k) const { return contains(IntVect{i, j, k}); }

  private:
    IntVect lo_{0, 0, 0}, hi_{-1, -1, -1};
};

AMREX_GPU_HOST_DEVICE inline constexpr Box grow(Box b, int n) { return b.grow(n); }

// ------------------------------------------------------------------ stencil view (engine hook)
template <class U> struct StencilView {
    const U* plane;  // shared memory: stencil-centre plane, pointing at (centre x, centre y), component 0
    const U* queue;  // registers: [2*qg + 1][qnc], slot (dk + qg) * qnc + n holds (centre x, centre y, k + dk)
    const U* glob;   // global memory: the centre cell, component 0
    Long gjs, gks, gns;
    int ci, cj, ck;
    int pjs, pns;    // shared-memory plane row and component strides
    int qg, qnc;     // register queue half-depth and component count
    int qrot = 0;    // circular queue (qlen > 0): offset k + dk sits in slot (dk + qg + qrot) % qlen
    int qlen = 0;
    const U* xw = nullptr; // registers: the centre row around the cell, [qnc][xwn], offset di at xw0 + di
    int xwn = 0, xw0 = 0;
#ifdef TREESAP_B200_CHECK
    // Checked builds: the valid index ranges of the shared-memory plane [plo, phi) and of the
    // global field [glo, ghi), relative to `plane` and `glob`; an access outside them sets bit 2
    // (index out of bounds) of the device error word `err` and reads the centre instead.
    int* err = nullptr;
    int plo = 0, phi = 0;
    Long glo = 0, ghi = 0;
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE void flag_bounds() const {
        if (!err) return;
#if defined(__CUDA_ARCH__)
        atomicOr(err, 2);
#else
        *err |= 2;
#endif
    }
#endif

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE const U& at(int i, int j, int k, int n) const {
        const int di = i - ci, dj = j - cj, dk = k - ck;
        if (xw != nullptr && dk == 0 && dj == 0 && xw0 + di >= 0 && xw0 + di < xwn && n < qnc)
            return xw[n * xwn + xw0 + di];
        if (dk == 0) {
            const int o = n * pns + dj * pjs + di;
#ifdef TREESAP_B200_CHECK
            if (o < plo || o >= phi) {
                flag_bounds();
                return plane[0];
            }
#endif
            return plane[o];
        }
        if (di == 0 && dj == 0 && dk >= -qg && dk <= qg && n < qnc) {
            const int m = dk + qg + qrot;
            return queue[(qlen > 0 ? m % qlen : m) * qnc + n];
        }
        const Long o = n * gns + dk * gks + dj * gjs + di;
#ifdef TREESAP_B200_CHECK
        if (o < glo || o >= ghi) {
            flag_bounds();
            return glob[0];
        }
#endif
        return glob[o];
    }
};

// ------------------------------------------------------------------ Array4
template <class T> struct Array4 {
    using value_type = std::remove_const_t<T>;

    T* AMREX_RESTRICT p = nullptr;
    Long jstride = 0, kstride = 0, nstride = 0;
    Dim3 begin{1, 1, 1}, end{0, 0, 0};
    int ncomp = 0;
    const StencilView<value_type>* view = nullptr;

    AMREX_GPU_HOST_DEVICE constexpr Array4() {}
    AMREX_GPU_HOST_DEVICE constexpr Array4(T* p_, Dim3 b, Dim3 e, int nc)
        : p(p_), jstride(e.x - b.x), kstride(Long(e.x - b.x) * (e.y - b.y)),
          nstride(Long(e.x - b.x) * (e.y - b.y) * (e.z - b.z)), begin(b), end(e), ncomp(nc) {}
    AMREX_GPU_HOST_DEVICE constexpr Array4(T* p_, Long js, Long ks, Long ns, Dim3 b, Dim3 e, int nc)
        : p(p_), jstride(js), kstride(ks), nstride(ns), begin(b), end(e), ncomp(nc) {}
    template <class U, class = std::enable_if_t<std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
    AMREX_GPU_HOST_DEVICE constexpr Array4(const Array4<U>& o)
        : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride), begin(o.begin), end(o.end),
          ncomp(o.ncomp), view(o.view) {}

    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T& operator()(int i, int j, int k, int n = 0) const {
        if constexpr (std::is_const_v<T>) {
            if (view) return view->at(i, j, k, n);
        }
        return p[(i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride];
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T& operator()(const IntVect& iv, int n = 0) const {
        return (*this)(iv[0], iv[1], iv[2], n);
    }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE T* ptr(int i, int j, int k, int n = 0) const {
        return p + ((i - begin.x) + (j - begin.y) * jstride + (k - begin.z) * kstride + n * nstride);
    }
    AMREX_GPU_HOST_DEVICE constexpr bool contains(int i, int j, int k) const {
        return i >= begin.x && i < end.x && j >= begin.y && j < end.y && k >= begin.z && k < end.z;
    }
    AMREX_GPU_HOST_DEVICE constexpr int nComp() const { return ncomp; }
};

// ------------------------------------------------------------------ geometry
namespace CoordSys {
enum CoordType { undef = -1, cartesian = 0, RZ = 1, SPHERICAL = 2 };
}

class RealBox {
  public:
    RealBox() = default;
    RealBox(const Array<Real, 3>& lo, const Array<Real, 3>& hi) : lo_(lo), hi_(hi) {}
    RealBox(Real x0, Real y0, Real z0, Real x1, Real y1, Real z1) : lo_{x0, y0, z0}, hi_{x1, y1, z1} {}
    Real lo(int d) const { return lo_[d]; }
    Real hi(int d) const { return hi_[d]; }
    Real length(int d) const { return hi_[d] - lo_[d]; }

  private:
    Array<Real, 3> lo_{0, 0, 0}, hi_{1, 1, 1};
};

struct GeometryData {
    GpuArray<Real, 3> prob_lo{}, prob_hi{}, dx{};
    Box domain{};
    int is_periodic[3] = {0, 0, 0};
    int coord = 0;
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE Real CellSize(int d) const { return dx[d]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE const Real* CellSize() const { return dx.data(); }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE Real ProbLo(int d) const { return prob_lo[d]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE Real ProbHi(int d) const { return prob_hi[d]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE const Box& Domain() const { return domain; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE int isPeriodic(int d) const { return is_periodic[d]; }
    AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE int Coord() const { return coord; }
};

class Geometry {
  public:
    Geometry() = default;
    // Same cell-size rule as AMReX: dx = (hi - lo) / number of cells.
    Geometry(const Box& dom, const RealBox* rb = nullptr, int coord = 0, int const* is_per = nullptr) {
        d_.domain = dom;
        d_.coord = coord;
        const RealBox r = rb ? *rb : RealBox{};
        for (int d = 0; d < 3; ++d) {
            d_.prob_lo[d] = r.lo(d);
            d_.prob_hi[d] = r.hi(d);
            d_.dx[d] = (r.hi(d) - r.lo(d)) / Real(dom.length(d));
            d_.is_periodic[d] = is_per ? (is_per[d] != 0) : 0;
        }
    }
    Geometry(const Box& dom, const RealBox& rb, int coord, const Array<int, 3>& is_per)
        : Geometry(dom, &rb, coord, is_per.data()) {}
    Real CellSize(int d) const { return d_.dx[d]; }
    GpuArray<Real, 3> CellSizeArray() const { return d_.dx; }
    GpuArray<Real, 3> InvCellSizeArray() const { return {1.0 / d_.dx[0], 1.0 / d_.dx[1], 1.0 / d_.dx[2]}; }
    GpuArray<Real, 3> ProbLoArray() const { return d_.prob_lo; }
    GpuArray<Real, 3> ProbHiArray() const { return d_.prob_hi; }
    Real ProbLo(int d) const { return d_.prob_lo[d]; }
    Real ProbHi(int d) const { return d_.prob_hi[d]; }
    const Box& Domain() const { return d_.domain; }
    bool isPeriodic(int d) const { return d_.is_periodic[d] != 0; }
    bool isAllPeriodic() const { return isPeriodic(0) && isPeriodic(1) && isPeriodic(2); }
    GeometryData data() const { return d_; }

  private:
    GeometryData d_;
};

// ------------------------------------------------------------------ boundary records
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
    AMREX_GPU_HOST_DEVICE constexpr BCRec() {}
    AMREX_GPU_HOST_DEVICE constexpr BCRec(int lx, int ly, int lz, int hx, int hy, int hz)
        : lo_{lx, ly, lz}, hi_{hx, hy, hz} {}
    AMREX_GPU_HOST_DEVICE constexpr int lo(int d) const { return lo_[d]; }
    AMREX_GPU_HOST_DEVICE constexpr int hi(int d) const { return hi_[d]; }

  private:
    int lo_[3] = {0, 0, 0}, hi_[3] = {0, 0, 0};
};

// ------------------------------------------------------------------ runtime stubs
inline void Initialize(int&, char**&, bool = true) {}
inline void Finalize() {}

struct PrintStream {
    template <class T> PrintStream& operator<<(const T& v) {
        std::cout << v;
        return *this;
    }
    PrintStream& operator<<(std::ostream& (*m)(std::ostream&)) {
        m(std::cout);
        return *this;
    }
};
inline PrintStream AllPrint() { return {}; }
inline PrintStream Print() { return {}; }

inline std::string Concatenate(const std::string& root, int num, int mindigits = 5) {
    std::string s = std::to_string(num);
    if (int(s.size()) < mindigits) s.insert(0, std::size_t(mindigits - int(s.size())), '0');
    return root + s;
}

} // namespace amrex
