// treesap-b200: named constant tensors (reference util/named_tensors.hpp:25-62).
#pragma once

namespace treesap {
namespace tensor {

/// Kronecker delta: 1 if a == b, else 0.
template <int a, int b> constexpr int kronecker = (a == b) ? 1 : 0;

namespace detail {
template <int... Indices> consteval int levi_civita_value() {
    constexpr int d = sizeof...(Indices);
    const int idx[] = {Indices...};
    for (int q = 0; q < d; ++q)
        if (idx[q] < 0 || idx[q] >= d) return 0;
    int inversions = 0;
    for (int p = 0; p < d; ++p)
        for (int q = p + 1; q < d; ++q) {
            if (idx[p] == idx[q]) return 0;
            if (idx[p] > idx[q]) ++inversions;
        }
    return (inversions % 2 == 0) ? 1 : -1;
}
} // namespace detail

/// Totally antisymmetric symbol in d = sizeof...(Indices) dimensions, indices 0..d-1:
/// +1 for even permutations of (0, .., d-1), -1 for odd ones, 0 otherwise.
template <int... Indices> constexpr int levi_civita = detail::levi_civita_value<Indices...>();

} // namespace tensor
} // namespace treesap
