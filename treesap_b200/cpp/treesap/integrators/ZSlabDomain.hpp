// treesap-b200: a domain split into z slabs, the block_size decomposition of
// SingleLevelIntegrator (reference SingleLevelIntegrator.hpp:47-49 and :172-176, where
// BoxArray::maxSize(block_size) chops the domain and FillPatch, :153-163, fills every box's
// ghost cells from its neighbours).
//
// Here the domain is cut along z only, into slabs of at most block_size[2] planes (near-equal
// depths; the stage kernels already tile x and y, so cutting them too would only add launches).
// Each slab is an ordinary single-box integrator (SingleLevelRK4Integrator,
// SingleLevelRK4F32StageIntegrator or SingleLevelEulerIntegrator) over its planes, with ngrow ghost planes on each side and the
// global geometry: the model sees global indices, the initial condition global coordinates.
// A step runs the slabs in lockstep, stage by stage:
//   1. every slab: stage register swap (the stage input becomes current);
//   2. every slab: halo exchange, then ghost fill. The exchange copies the valid x-y region
//      of the neighbouring slabs' ngrow boundary planes (same stage register) into the slab's
//      ghost planes (periodic in z: the first and last slabs are neighbours); the ghost fill
//      then completes every other ghost cell, with global coordinates and the periodic
//      images of the slab's own planes (exchange planes included);
//   3. every slab: the fused stage kernel.
// Every ghost cell therefore holds what the single box would hold, and the result is bitwise
// the single-box result. All slabs share the context's stream and device; a rank of a
// multi-GPU run holds its own slabs and exchanges its outer faces through the C ABI
// (ts_slab_*), see treesap_b200/slabs.py.
#pragma once

#include <memory>
#include <stdexcept>
#include <vector>

#include "../SingleLevelIntegrator.hpp"

namespace treesap {

/// Near-equal split of nz planes into ceil(nz / block) slabs (depths differ by at most one).
/// Returns the first plane of each slab and nz at the end.
inline std::vector<int> zslab_bounds(int nz, int block) {
    if (block < 1) throw std::invalid_argument("block_size must be positive");
    const int n = (nz + block - 1) / block;
    std::vector<int> b(n + 1);
    for (int k = 0; k <= n; ++k) b[k] = int((long long)nz * k / n);
    return b;
}

template <class Integ> class ZSlabDomain {
  public:
    using Model = std::decay_t<decltype(std::declval<const Integ&>().get_model())>;
    static constexpr int ncomp = Model::ncomp;
    static constexpr int ngrow = Model::ngrow;
    using Field = treesap_b200::DeviceField<amrex::Real>;

    ZSlabDomain(Model model, const amrex::IntVect& block_size, ts_context* ctx = nullptr) {
        const amrex::GeometryData g = model.get_geometry().data();
        nz_ = g.domain.length(2);
        nxy_ = (long long)g.domain.length(0) * g.domain.length(1);
        periodic_z_ = g.is_periodic[2] != 0;
        bounds_ = zslab_bounds(nz_, block_size[2]);
        const int n = int(bounds_.size()) - 1;
        for (int k = 0; k < n; ++k)
            if (bounds_[k + 1] - bounds_[k] < ngrow)
                throw std::invalid_argument("z slabs thinner than the ghost width (block_size[2] too small)");
        for (int k = 0; k < n; ++k) {
            treesap_b200::SlabZ sz;
            sz.zoff = bounds_[k];
            sz.nz = nz_;
            sz.lo_ex = n > 1 && (k > 0 || periodic_z_);
            sz.hi_ex = n > 1 && (k < n - 1 || periodic_z_);
            slabs_.push_back(std::make_unique<Integ>(model, block_size, ctx, sz, bounds_[k + 1] - bounds_[k]));
        }
        for (int k = 0; k < n; ++k)
            slabs_[k]->set_halo_hook([this, k](const typename Integ::FieldRef& f) { exchange(k, f); });
        dt_ = model.dt_hint();
    }

    int slabs() const { return int(slabs_.size()); }
    Integ& slab(int k) { return *slabs_[k]; }
    const std::vector<int>& bounds() const { return bounds_; }

    void initialise() {
        for (auto& s : slabs_) s->initialise();
    }

    /// One step of every slab in lockstep, stage by stage.
    void step() {
        for (int st = 0; st < Integ::kStages; ++st) {
            for (auto& s : slabs_) s->stage_prepare(st);
            for (auto& s : slabs_) s->stage_fill(st, dt_);
            for (auto& s : slabs_) s->stage_launch(st, dt_);
        }
        for (auto& s : slabs_) s->stage_finish(dt_);
    }

    /// The valid state of the whole domain, [comp][z][y][x] (host or device memory).
    void set_state(const double* src, bool src_on_device = false) {
        with_slab_buffers(src_on_device, [&](int k, double* buf, long long ncell) {
            gather(src, buf, k, ncell, true, src_on_device);
            slabs_[k]->set_state(buf, src_on_device);
        });
    }
    void get_state(double* dst, bool dst_on_device = false) {
        with_slab_buffers(dst_on_device, [&](int k, double* buf, long long ncell) {
            slabs_[k]->get_state(buf, dst_on_device);
            gather(dst, buf, k, ncell, false, dst_on_device);
        });
    }

    double time() const { return slabs_.front()->get_time(); }
    long long steps() const { return (long long)slabs_.front()->get_steps(); }
    long long launches_per_step() const {
        long long n = 0;
        for (auto& s : slabs_) n += s->launches_per_step();
        return n;
    }
    bool state_is_finite() {
        bool ok = true;
        for (auto& s : slabs_) ok = s->state_is_finite() && ok;
        return ok;
    }
    void set_launch_shape(int rows, int chunks) {
        for (auto& s : slabs_) s->set_launch_shape(rows, chunks);
    }
    void attach_clock(KernelClock* c) {
        for (auto& s : slabs_) s->attach_clock(c);
    }

  private:
    /// Halo exchange into the ghost planes of slab k's field f from the neighbours' current stage
    /// input (the valid x-y region of their ngrow boundary planes).
    void exchange(int k, const typename Integ::FieldRef& f) {
        const int n = slabs();
        const treesap_b200::SlabZ& sz = slabs_[k]->slab();
        const int depth = bounds_[k + 1] - bounds_[k];
        Integ& me = *slabs_[k];
        const int st = stage_of(me, f.data);
        if (sz.lo_ex) {
            const int kn = (k + n - 1) % n;
            copy_planes(me, f, -ngrow, slabs_[kn]->stage_ref(st), bounds_[kn + 1] - bounds_[kn] - ngrow);
        }
        if (sz.hi_ex) copy_planes(me, f, depth, slabs_[(k + 1) % n]->stage_ref(st), 0);
    }

    /// ngrow planes from plane `ks0` of `src` into planes [kd0, kd0 + ngrow) of `dst`.
    static void copy_planes(Integ& me, const typename Integ::FieldRef& dst, int kd0, const typename Integ::FieldRef& src,
                            int ks0) {
        const auto& Ls = src.L;
        const long long off = (long long)(ks0 + ngrow) * Ls.px * Ls.py;
        if (dst.L.esize == 8)
            treesap_b200::launch_halo_copy(static_cast<double*>(dst.data), dst.L, kd0,
                                           static_cast<const double*>(src.data) + off, Ls.comp_stride(), ngrow,
                                           me.sm_count(), me.stream());
        else
            treesap_b200::launch_halo_copy(static_cast<float*>(dst.data), dst.L, kd0,
                                           static_cast<const float*>(src.data) + off, Ls.comp_stride(), ngrow,
                                           me.sm_count(), me.stream());
    }

    /// Which stage register `data` is (the neighbours' register of the same stage is the source).
    static int stage_of(Integ& me, const void* data) {
        for (int st = Integ::kStages - 1; st >= 0; --st)
            if (me.stage_ref(st).data == data) return st;
        return 0;
    }

    /// Per slab: a buffer of its valid cells ([comp][z_slab][y][x]) in the memory kind of the
    /// caller's array.
    template <class F> void with_slab_buffers(bool device, F&& f) {
        for (int k = 0; k < slabs(); ++k) {
            const long long ncell = nxy_ * (bounds_[k + 1] - bounds_[k]);
            const size_t bytes = sizeof(double) * size_t(ncell) * ncomp;
            if (device) {
                double* buf = nullptr;
                treesap_b200::cuda_check(cudaMalloc(&buf, bytes), "cudaMalloc(slab buffer)");
                try {
                    f(k, buf, ncell);
                } catch (...) {
                    cudaFree(buf);
                    throw;
                }
                treesap_b200::cuda_check(cudaStreamSynchronize(slabs_[k]->stream()), "cudaStreamSynchronize");
                cudaFree(buf);
            } else {
                std::vector<double> buf(size_t(ncell) * ncomp);
                f(k, buf.data(), ncell);
            }
        }
    }

    /// Copies slab k's part of a whole-domain array to (to_slab) or from its slab buffer.
    void gather(const double* whole_src, double* buf, int k, long long ncell, bool to_slab, bool device) const {
        const long long dom = nxy_ * nz_;
        const size_t bytes = sizeof(double) * size_t(ncell);
        for (int c = 0; c < ncomp; ++c) {
            const double* a = whole_src + c * dom + nxy_ * bounds_[k];
            double* w = const_cast<double*>(a);
            double* b = buf + c * ncell;
            if (device) {
                treesap_b200::cuda_check(cudaMemcpyAsync(to_slab ? b : w, to_slab ? a : b, bytes, cudaMemcpyDeviceToDevice,
                                                         slabs_[k]->stream()),
                                         "cudaMemcpyAsync(slab gather)");
            } else {
                std::memcpy(to_slab ? b : w, to_slab ? a : b, bytes);
            }
        }
    }
    void gather(double* whole_dst, double* buf, int k, long long ncell, bool to_slab, bool device) const {
        gather(static_cast<const double*>(whole_dst), buf, k, ncell, to_slab, device);
    }

    std::vector<std::unique_ptr<Integ>> slabs_;
    std::vector<int> bounds_;
    int nz_ = 0;
    long long nxy_ = 0;
    bool periodic_z_ = false;
    amrex::Real dt_ = 0.0;
};

} // namespace treesap
