// treesap-b200: initial condition from run-time expressions of x, y, z, one per component
// (reference init/FunctionInit.hpp:34-101, which compiles amrex::Parser objects).
//
// The constructor compiles each expression on the host (util/expression.hpp) and keeps the
// programs in a process-wide registry, one host copy and (in CUDA builds) one device copy that
// live until exit, like the reference's static parser registry; the functor itself holds
// only pointers and stays trivially copyable, so it travels into the init kernel by value.
#pragma once

#include <AMReX.H>

#include <deque>
#include <mutex>
#include <string>
#include <vector>

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

#include "../pde-model/PDEModelConcepts.hpp"
#include "../util/expression.hpp"

namespace treesap {

namespace detail {
/// A compiled program with a stable host copy and, in CUDA builds, a device copy.
struct ExprProgram {
    const expr::Instr* host = nullptr;
    const expr::Instr* device = nullptr;
    int size = 0;
};

inline ExprProgram register_expression(const std::string& text) {
    static std::mutex m;
    static std::deque<std::vector<expr::Instr>> host_programs;
    std::vector<expr::Instr> code = expr::Compiler::compile(text);
    std::lock_guard<std::mutex> lock(m);
    host_programs.push_back(std::move(code));
    const auto& h = host_programs.back();
    ExprProgram p;
    p.host = h.data();
    p.size = int(h.size());
#if defined(__CUDACC__)
    void* d = nullptr;
    if (cudaMalloc(&d, sizeof(expr::Instr) * (h.size() ? h.size() : 1)) != cudaSuccess ||
        cudaMemcpy(d, h.data(), sizeof(expr::Instr) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("FunctionInit: device copy of the expression failed");
    p.device = static_cast<const expr::Instr*>(d);
#else
    p.device = p.host;
#endif
    return p;
}
} // namespace detail

template <int ncomp_> struct FunctionInit {
    static_assert(ncomp_ > 0, "FunctionInit must initialise a positive number of components.");
    static constexpr int ncomp = ncomp_;

    FunctionInit() = delete;

    /// Compiles one expression of x, y, z per component (invalid text throws std::invalid_argument).
    explicit FunctionInit(const amrex::Array<std::string, ncomp>& exprs) {
        for (int i = 0; i < ncomp; ++i) programs[i] = detail::register_expression(exprs[i]);
    }

    template <int comp>
    AMREX_GPU_HOST_DEVICE amrex::Real operator()(amrex::Real x, amrex::Real y, amrex::Real z) const {
        const detail::ExprProgram& p = programs[comp];
#if defined(__CUDA_ARCH__)
        return expr::eval(p.device, p.size, x, y, z);
#else
        return expr::eval(p.host, p.size, x, y, z);
#endif
    }

  private:
    detail::ExprProgram programs[ncomp];
};

static_assert(InitConcept<FunctionInit<1>>);

} // namespace treesap
