// treesap-b200 (no reference implementation; the adaptive scheme the reference's
// computeNewState(dt_hint) contract anticipates, SingleLevelIntegrator.hpp:128-142 and
// PDEModel.hpp:115-122 of the reference): Dormand-Prince 5(4) with step-size control.
//
// The embedded Runge-Kutta pair of Dormand & Prince (1980), 7 stages:
//   K_s = F(t + c_s dt, y + dt sum_{j<s} a_sj K_j),   s = 0..6,
//   y_new = y + dt sum_j b_j K_j   (5th order; the argument of stage 6, so K_6 = F(y_new)),
//   err_c = dt sum_j e_j K_j       (e = b - b*, the difference to the embedded 4th-order solution).
// Each stage is one fused stage kernel whose epilogue (EpiDP<s>) stores K_s and forms the next
// stage's argument from y and K_0..K_s at the same cell; stage 6's epilogue reduces the scaled
// error max_{cells, comps} |err_c| / (atol + rtol max(|y|, |y_new|)) into one device word. The
// host accepts the step when the error is <= 1 and proposes dt_new = dt min(5, max(0.2,
// 0.9 err^{-1/5})) (Hairer, Norsett & Wanner, Solving ODEs I, II.4); a rejected step is retried
// from y with the smaller dt. computeNewState returns the dt taken. Every attempt runs all 7
// stage kernels: reusing K_6 = F(y_new) as the next K_0 (first-same-as-last) would need a
// separate kernel to form the first stage argument, which stage 0's epilogue provides here.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "../SingleLevelIntegrator.hpp"

namespace treesap_b200 {

/// Dormand-Prince 5(4) coefficients (Dormand & Prince 1980): c_s, the rows a(s, j) (j < s; row 6
/// is b), and e_j = b_j - b*_j (the 4th-order weights b* subtracted). Constant-folded wherever
/// the indices are compile-time constants (the stage epilogues' unrolled loops).
struct DP5 {
    AMREX_GPU_HOST_DEVICE static constexpr double c(int s) {
        constexpr double t[7] = {0.0, 1.0 / 5.0, 3.0 / 10.0, 4.0 / 5.0, 8.0 / 9.0, 1.0, 1.0};
        return t[s];
    }
    AMREX_GPU_HOST_DEVICE static constexpr double a(int s, int j) {
        constexpr double t[7][6] = {
            {0, 0, 0, 0, 0, 0},
            {1.0 / 5.0, 0, 0, 0, 0, 0},
            {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
            {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
            {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
            {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
            {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
        return t[s][j];
    }
    AMREX_GPU_HOST_DEVICE static constexpr double e(int j) {
        constexpr double t[7] = {71.0 / 57600.0,      0.0,         -71.0 / 16695.0, 71.0 / 1920.0,
                                 -17253.0 / 339200.0, 22.0 / 525.0, -1.0 / 40.0};
        return t[j];
    }
};

/// Epilogue of Dormand-Prince stage S: stores K_S, and for S < 6 the next stage argument
/// y + dt sum_{j<=S} a[S+1][j] K_j (K_j, j < S, and y read at the cell from global memory); for
/// S = 6 (input y_new) the scaled error max into *err_max (the bits of a non-negative double,
/// which order like unsigned integers).
template <int S> struct EpiDP : NoCentre {
    struct Params {
        double* k[7];
        const double* y;
        double* next;   // S < 6: the next stage argument (S = 5: y_new)
        Layout L;
        double dt;
        double atol, rtol;
        unsigned long long* err_max;
    };
    template <class T, int NC, int CX, class CO>
    static __device__ __forceinline__ void apply(const Params& p, const T (&k)[CX][NC], const bool (&act)[CX],
                                                 const T* centre, int pns, int i0, int j, int z, const CO&) {
        const long long cs = p.L.comp_stride();
        double emax = 0.0;
#pragma unroll
        for (int e = 0; e < CX; ++e) {
            if (!act[e]) continue;
            const long long o = p.L.index(i0 + e, j, z, 0);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const long long oc = o + c * cs;
                const double ks = double(k[e][c]);
                p.k[S][oc] = ks;
                const double yv = p.y[oc];
                if constexpr (S < 6) {
                    double acc = 0.0;
                    treesap::static_for<0, S>([&]<int q>() {
                        if constexpr (DP5::a(S + 1, q) != 0.0) acc += DP5::a(S + 1, q) * p.k[q][oc];
                    });
                    acc += DP5::a(S + 1, S) * ks;
                    p.next[oc] = yv + p.dt * acc;
                } else {
                    double err = 0.0;
                    treesap::static_for<0, 6>([&]<int q>() {
                        if constexpr (DP5::e(q) != 0.0) err += DP5::e(q) * p.k[q][oc];
                    });
                    err += DP5::e(6) * ks;
                    const double ynew = double(centre[c * pns + e]);
                    const double scale = p.atol + p.rtol * fmax(fabs(yv), fabs(ynew));
                    emax = fmax(emax, fabs(p.dt * err) / scale);
                }
            }
        }
        if constexpr (S == 6) {
            // non-finite errors count as a failed step (NaN would not compare)
            if (!(emax <= 1e300)) emax = 1e300;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, off));
            if ((threadIdx.x & 31) == 0 && emax > 0.0)
                atomicMax(p.err_max, static_cast<unsigned long long>(__double_as_longlong(emax)));
        }
    }
};

} // namespace treesap_b200

namespace treesap {

template <typename PDEModelType>
    requires PDEModelConcept<PDEModelType>
class SingleLevelDOPRI5Integrator : public SingleLevelIntegrator<PDEModelType> {
    using Base = SingleLevelIntegrator<PDEModelType>;
    using Base::FillPatch;
    using Base::geom;
    using Base::model;
    using Base::ncomp;
    using Base::ngrow;
    using Base::state_new;
    using Base::state_old;
    using Base::time;
    using typename Base::Field;
    using typename Base::RHSType;

  public:
    using Tile = typename detail::DefaultTile<double, ngrow, ncomp>::type;

    /// rtol, atol: the error tolerances of the step-size control.
    SingleLevelDOPRI5Integrator(PDEModelType model_, const amrex::IntVect& block_size, ts_context* ctx_ = nullptr,
                                double rtol = 1e-6, double atol = 1e-9)
        : Base(std::move(model_), block_size, ctx_), k{Field(this->extent(), ngrow, ncomp), Field(this->extent(), ngrow, ncomp),
                                                        Field(this->extent(), ngrow, ncomp), Field(this->extent(), ngrow, ncomp),
                                                        Field(this->extent(), ngrow, ncomp), Field(this->extent(), ngrow, ncomp),
                                                        Field(this->extent(), ngrow, ncomp)},
          argA(this->extent(), ngrow, ncomp), argB(this->extent(), ngrow, ncomp), rtol_(rtol), atol_(atol) {
        if (!(rtol > 0.0) || !(atol > 0.0)) throw std::invalid_argument("DOPRI5 tolerances must be positive");
        treesap_b200::cuda_check(cudaMalloc(&err_dev, sizeof(unsigned long long)), "cudaMalloc(error max)");
        treesap_b200::cuda_check(cudaMallocHost(&err_host, sizeof(unsigned long long)), "cudaMallocHost(error max)");
    }
    ~SingleLevelDOPRI5Integrator() override {
        if (err_dev) cudaFree(err_dev);
        if (err_host) cudaFreeHost(err_host);
    }

    /// Steps accepted and rejected so far, and the step size proposed for the next step.
    long long accepted() const { return accepted_; }
    long long rejected() const { return rejected_; }
    double proposed_dt() const { return dt_next_; }
    /// The scaled error norm of the last attempted step.
    double last_error() const { return last_err_; }

    void initialise_impl() override {
        Base::initialise_impl();
        dt_next_ = 0.0;
        accepted_ = rejected_ = 0;
    }

  protected:
    amrex::Real computeNewState(amrex::Real dt_hint) override {
        if (this->dry_run_) throw std::invalid_argument("adaptive steps cannot be replayed from a graph");
        if (this->steps == 0 || !(dt_next_ > 0.0)) {
            // a fresh run (initialise or set_state): start from the model's dt and clear the counts
            dt_next_ = dt_hint;
            accepted_ = rejected_ = 0;
        }
        for (int attempt = 0; attempt < 64; ++attempt) {
            const double dt = dt_next_;
            const double err = attempt_step(dt);
            last_err_ = err;
            const double fac = err > 0.0 ? 0.9 * std::pow(err, -0.2) : 5.0;
            if (err <= 1.0) {
                dt_next_ = dt * std::min(5.0, std::max(0.2, fac));
                ++accepted_;
                this->launches_per_step_ = launches_;
                return dt;
            }
            ++rejected_;
            dt_next_ = dt * std::max(0.2, std::min(1.0, fac));
        }
        throw std::runtime_error("DOPRI5: step size control failed (64 rejected attempts)");
    }

  private:
    /// One attempted step of width dt from y = state_old: the scaled error norm.
    double attempt_step(double dt) {
        launches_ = this->fills_this_step_;
        treesap_b200::cuda_check(cudaMemsetAsync(err_dev, 0, sizeof(unsigned long long), this->stream()),
                                 "cudaMemsetAsync(error max)");
        // stage inputs: y, A, B, A, B, A, y_new (state_new)
        Field* in = &state_old;
        Field* out = &argA;
        for (int s = 0; s < 7; ++s) {
            if (s > 0) {
                if (s == 6) in = &state_new;
                FillPatch(*in, time + DP5c(s) * dt);
            }
            Field* next = s == 5 ? &state_new : out;
            launch(s, *in, next, dt);
            if (s < 6) {
                in = next;
                out = (next == &argA) ? &argB : &argA;
            }
        }
        treesap_b200::cuda_check(cudaMemcpyAsync(err_host, err_dev, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                                 this->stream()),
                                 "cudaMemcpyAsync(error max)");
        treesap_b200::cuda_check(cudaStreamSynchronize(this->stream()), "cudaStreamSynchronize(error max)");
        double err;
        std::memcpy(&err, err_host, sizeof(double));
        return err;
    }

    static double DP5c(int s) { return treesap_b200::DP5::c(s); }

    void launch(int s, const Field& input, Field* next, double dt) {
        switch (s) {
        case 0: launch_stage<0>(input, next, dt); break;
        case 1: launch_stage<1>(input, next, dt); break;
        case 2: launch_stage<2>(input, next, dt); break;
        case 3: launch_stage<3>(input, next, dt); break;
        case 4: launch_stage<4>(input, next, dt); break;
        case 5: launch_stage<5>(input, next, dt); break;
        default: launch_stage<6>(input, next, dt); break;
        }
        ++launches_;
    }

    template <int S> void launch_stage(const Field& input, Field* next, double dt) {
        using namespace treesap_b200;
        const Layout& L = input.layout();
        StageParams<double> sp{};
        sp.in = input.data();
        sp.L = L;
        sp.geom = geom;
        sp.time = time + DP5::c(S) * dt;
        sp.err = ts_context_error_word(this->ctx);
        typename EpiDP<S>::Params ep{};
        for (int q = 0; q < 7; ++q) ep.k[q] = k[q].data();
        ep.y = state_old.data();
        ep.next = S < 6 ? next->data() : nullptr;
        ep.L = L;
        ep.dt = dt;
        ep.atol = atol_;
        ep.rtol = rtol_;
        ep.err_max = err_dev;
        using Launcher = StageLauncher<Tile, RHSType, EpiDP<S>>;
        const auto shape = Launcher::shape(L, this->sm_count(), this->tile_rows, this->z_chunks);
        const CUtensorMap& tm = this->tensor_map(input.data(), L, TS_F64, Launcher::box_x(), Launcher::box_y(shape));
        const CentreMaps cm = this->template centre_maps<Launcher>(ep, shape);
        this->take_stage_fault(sp);
        this->clock_begin(1 + (S < 4 ? S : 3));
        Launcher::launch(tm, cm, sp, model.get_rhs(), ep, shape, this->stream());
        this->clock_end();
    }

    Field k[7];
    Field argA, argB;
    double rtol_, atol_;
    unsigned long long* err_dev = nullptr;
    unsigned long long* err_host = nullptr;
    double dt_next_ = 0.0;
    double last_err_ = 0.0;
    long long accepted_ = 0, rejected_ = 0, launches_ = 0;
};

} // namespace treesap
