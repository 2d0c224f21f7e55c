// Test driver for clwilson_b200/csrc/wl_plan.h (dense split boundaries), used
// by tests/test_split_plan.py.  Prints, for class target T, dense limit qd and
// Sd splits: the grid size, then one line per boundary k = 1 .. Sd-1 with its q
// and the model's cumulative cost at q (interpolated like the boundary).
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include "wl_plan.h"

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const double T = atof(argv[1]), qd = atof(argv[2]);
    const uint64_t Sd = strtoull(argv[3], nullptr, 0);
    std::vector<double> grid, cum;
    double cols = 0;
    dense_cost_grid(T, qd, grid, cum, &cols);
    printf("grid %zu total %.17g\n", grid.size(), cum.back());
    for (uint64_t k = 1; k < Sd; ++k) {
        const double q = dense_boundary(grid, cum, k, Sd);
        // cumulative cost at q, linear between grid points
        size_t j = std::upper_bound(grid.begin(), grid.end(), q) - grid.begin();
        double c = cum.back();
        if (j > 0 && j < grid.size())
            c = cum[j - 1] + (cum[j] - cum[j - 1]) * (q - grid[j - 1]) / (grid[j] - grid[j - 1]);
        printf("%.17g %.17g\n", q, c);
    }
    return 0;
}
