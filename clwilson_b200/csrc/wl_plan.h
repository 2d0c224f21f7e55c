// wl_plan.h -- the cost model behind the dense sweep's split boundaries.
// Host code only (no CUDA).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

// Cells per row that a dense column at prime q costs for class target T: one
// for the prefix product plus 7/8 of one per 3-bit window of the exponent's
// low part, s ~ log2(8 T ln(q) / q^2) bits when the high part changes every 8
// columns (k_sweep_dense), at most the exponent's length.
inline double dense_cells_at(double T, double q) {
    const double e = T / (q - 1.0);
    double sb = std::log2(std::max(1.0, 8.0 * T * std::log(q) / (q * q)));
    sb = std::min(sb, std::log2(std::max(e, 1.0)) + 1.0);
    return 1.0 + 0.875 * std::ceil(sb / 3.0);
}

// Cumulative dense cost over q in [2, qd] on a log grid: cum[k] for q = grid[k].
inline void dense_cost_grid(double T, double qd, std::vector<double>& grid, std::vector<double>& cum, double* cols_est) {
    const int N = 2048;
    grid.assign(N + 1, 0.0);
    cum.assign(N + 1, 0.0);
    const double u0 = std::log(2.0), u1 = std::log(std::max(qd, 3.0));
    const double du = (u1 - u0) / N;
    double c = 0, n = 0;
    grid[0] = 2.0;
    for (int k = 1; k <= N; ++k) {
        const double u = u0 + (k - 0.5) * du, q = std::exp(u);
        const double dn = q * du / u;            // primes in the step ~ dq / ln q
        n += dn;
        c += dn * dense_cells_at(T, q);
        grid[k] = std::exp(u0 + k * du);
        cum[k] = c;
    }
    *cols_est = n;
}

// Value of q where dense split k of Sd ends: the point of equal cumulative
// cost k/Sd, interpolated inside a grid step (there are more splits than grid
// points when the dense region is long, and a boundary snapped to the grid
// would leave empty splits next to ones many times too long).  Inside a step
// the cost per unit of ln q grows about like q, so the interpolation is linear
// in q between the grid points.
inline double dense_boundary(const std::vector<double>& grid, const std::vector<double>& cum, uint64_t k, uint64_t Sd) {
    const double target = cum.back() * (double)k / (double)Sd;
    size_t j = std::lower_bound(cum.begin(), cum.end(), target) - cum.begin();
    if (j >= cum.size()) j = cum.size() - 1;
    double q = grid[j];
    if (j > 0 && cum[j] > cum[j - 1]) {
        const double f = (target - cum[j - 1]) / (cum[j] - cum[j - 1]);
        q = grid[j - 1] + f * (grid[j] - grid[j - 1]);
    }
    return q;
}
