// treesap-b200: compile-time integer and rational helpers used for stencil weights.
// Public API of the reference util/cexprmath.hpp:32-105 (factorial, binom, power,
// alternating_sign, generalised_harmonic_number), device-callable.
#pragma once

#include <AMReX.H>

#include <cstdint>

namespace treesap {
namespace cexprmath {

/// n! (exact in 64 bits for n <= 20).
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr std::int64_t factorial(int n) {
    std::int64_t f = 1;
    while (n > 1) f *= n--;
    return f;
}

/// Binomial coefficient C(n, k); 0 outside 0 <= k <= n.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr std::int64_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    const int m = (k < n - k) ? k : n - k;
    std::int64_t c = 1;
    for (int q = 0; q < m; ++q) c = c * (n - q) / (q + 1); // exact: c * (n-q) is divisible by q+1
    return c;
}

/// base^exponent for exponent >= 0.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr std::int64_t power(std::int64_t base, int exponent) {
    std::int64_t r = 1;
    for (int q = 0; q < exponent; ++q) r *= base;
    return r;
}

/// (-1)^k.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr int alternating_sign(int k) { return (k % 2 == 0) ? 1 : -1; }

/// H_{n,m} = sum_{k=1..n} 1/k^m, summed in increasing k.
AMREX_GPU_HOST_DEVICE AMREX_FORCE_INLINE constexpr double generalised_harmonic_number(int n, int m) {
    double h = 0.0;
    for (int k = 1; k <= n; ++k) h += 1.0 / static_cast<double>(power(k, m));
    return h;
}

} // namespace cexprmath
} // namespace treesap
