// batch_plan.h -- work units of the persistent batch kernel (batch.cu).
//
// Pure host code (no CUDA), so the plan's invariants are tested on the CPU
// (tests/batch_plan_harness.cpp): unit boundaries are non-decreasing tile
// indices from 0 to the tile count, unit u's first job holds its first
// tile, and every unit's cost stays within one tile of the average.
#pragma once

#include <algorithm>
#include <vector>

namespace rsgpu {

struct BatchUnitPlan {
    std::vector<long long> unit_first;  // n_units + 1 entries: unit u is tiles [unit_first[u], unit_first[u+1])
    std::vector<int> unit_job;          // the job holding tile unit_first[u]
};

// Jobs in order: job i holds tiles [tile_begin[i], tile_begin[i] + tiles[i])
// (consecutive, tiles[i] >= 1) and costs cost[i], spread evenly over its
// tiles.  Units are cut where the running cost crosses u/n_units of the
// total, so each unit costs the average to within one tile.
inline BatchUnitPlan plan_batch_units(const std::vector<long long> &tile_begin, const std::vector<long long> &tiles,
                                      const std::vector<double> &cost, int n_units) {
    BatchUnitPlan p;
    const size_t n = tile_begin.size();
    const long long t = n ? tile_begin[n - 1] + tiles[n - 1] : 0;
    double total = 0;
    for (double c : cost) total += c;
    n_units = std::max(1, n_units);
    p.unit_first.assign(n_units + 1, t);
    p.unit_first[0] = 0;
    double acc = 0;
    int unit = 1;
    for (size_t i = 0; i < n && unit < n_units; i++) {
        const double per_tile = cost[i] / (double)tiles[i];
        for (long long k = 0; k < tiles[i] && unit < n_units; k++) {
            acc += per_tile;
            while (unit < n_units && acc >= total * unit / n_units) p.unit_first[unit++] = tile_begin[i] + k + 1;
        }
    }
    for (int u = 1; u <= n_units; u++) p.unit_first[u] = std::max(p.unit_first[u], p.unit_first[u - 1]);
    p.unit_first[n_units] = t;
    p.unit_job.assign(n_units, 0);
    size_t jj = 0;
    for (int u = 0; u < n_units; u++) {
        while (jj + 1 < n && tile_begin[jj + 1] <= p.unit_first[u]) jj++;
        p.unit_job[u] = (int)jj;
    }
    return p;
}

}  // namespace rsgpu
