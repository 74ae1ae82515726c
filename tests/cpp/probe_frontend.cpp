// Host-side probe of the treesap-b200 header front end (compiled by tests/test_frontend.py with
// g++; no CUDA needed): prints the stencil weights, Kreiss-Oliger coefficients and tensor-alias
// index maps as JSON, and checks the compile-time API surface.
#include <cstdio>

#include "pde-model/tensor-alias/RankNAlias.hpp"
#include "pde-model/tensor-alias/SymRank2Alias.hpp"
#include "util/cexprmath.hpp"
#include "util/named_tensors.hpp"
#include "util/stencil.hpp"
#include "util/tensor_operations.hpp"

using namespace treesap;

template <int n> void weights(const char* sep) {
    std::printf("\"%d\": {\"first\": [", n);
    for (int p = 0; p <= n; ++p) std::printf("%s%.17g", p ? ", " : "", stencil_impl::weights::first<n>(p));
    std::printf("], \"second\": [");
    for (int p = 0; p <= n; ++p) std::printf("%s%.17g", p ? ", " : "", stencil_impl::weights::second<n>(p));
    std::printf("], \"third\": [");
    if constexpr (n >= 2)
        for (int p = 0; p <= n; ++p) std::printf("%s%.17g", p ? ", " : "", stencil_impl::weights::third<n>(p));
    std::printf("], \"ko\": [");
    for (int s = 0; s <= n; ++s)
        std::printf("%s%lld", s ? ", " : "",
                    (long long)(-cexprmath::alternating_sign(s) * cexprmath::binom(2 * n, n + s)));
    std::printf("]}%s\n", sep);
}

int main() {
    static_assert(tensor::kronecker<1, 1> == 1 && tensor::kronecker<0, 2> == 0);
    static_assert(tensor::levi_civita<0, 1, 2> == 1 && tensor::levi_civita<1, 0, 2> == -1 &&
                  tensor::levi_civita<0, 0, 2> == 0 && tensor::levi_civita<2, 0, 1> == 1);
    static_assert(tensor::contract<2, 2>([]<int a, int b>() { return a * 10 + b; }) == 22);
    static_assert(tensor::contract([]<int a>() { return a; }) == 3);
    std::printf("{\"weights\": {\n");
    weights<1>(",");
    weights<2>(",");
    weights<3>(",");
    weights<4>("");
    std::printf("}, \"sym2\": [");
    using S = tensor::SymRank2Alias<6>;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            std::printf("%s[%d, %d, %d]", (a || b) ? ", " : "", a, b, S::get_absolute({a, b}));
    std::printf("], \"rank2\": [");
    using R2 = tensor::Rank2Alias<1>;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            std::printf("%s[%d, %d, %d]", (a || b) ? ", " : "", a, b, R2::get_absolute({a, b}));
    std::printf("]}\n");
    return 0;
}
