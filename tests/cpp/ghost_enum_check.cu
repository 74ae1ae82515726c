// Host-only check of the ghost-cell enumeration of the fill kernels (engine/grid_kernels.cuh
// ghost_coords): for every layout below, ghost index t = 0 .. count-1 visits every ghost cell of
// the box grown by the ghost width exactly once and no valid cell. Exit status 0 = pass.
#include <cstdio>
#include <set>
#include <tuple>
#include "engine/grid_kernels.cuh"
using namespace treesap_b200;
int main() {
    int fails = 0;
    const int sizes[][3] = {{3, 2, 5}, {16, 16, 16}, {37, 29, 41}, {1, 1, 7}, {4, 5, 4}, {64, 8, 40}, {96, 96, 96}};
    for (auto& n : sizes)
        for (int g = 1; g <= 4; ++g) {
            Layout L = Layout::make(n, g, 2, 8);
            const long long tot = ghost_count(L).total();
            std::set<std::tuple<int, int, int>> seen;
            for (long long t = 0; t < tot; ++t) {
                int i, j, k;
                ghost_coords(L, t, i, j, k);
                bool inside = i >= 0 && i < n[0] && j >= 0 && j < n[1] && k >= 0 && k < n[2];
                bool inrange = i >= -g && i < n[0] + g && j >= -g && j < n[1] + g && k >= -g && k < n[2] + g;
                if (inside || !inrange || !seen.insert({i, j, k}).second) { ++fails; break; }
            }
            const long long want = (long long)(n[0] + 2 * g) * (n[1] + 2 * g) * (n[2] + 2 * g) - (long long)n[0] * n[1] * n[2];
            if ((long long)seen.size() != want) ++fails;
        }
    printf("fails %d\n", fails);
    return fails != 0;
}
