// Work units of the persistent batch kernel (reedsolomon_b200/csrc/
// batch_plan.h), checked on the CPU over random job lists: boundaries run
// from tile 0 to the tile count without decreasing, each unit's first job
// holds its first tile, and no unit costs more than the average plus one
// tile (units are cut at the first tile where the running cost reaches
// their share).
#include <cmath>
#include <cstdio>
#include <random>

#include "batch_plan.h"

int main() {
    std::mt19937_64 rng(777);
    for (int it = 0; it < 3000; it++) {
        const int n = 1 + (int)(rng() % 3000);
        std::vector<long long> begin(n), tiles(n);
        std::vector<double> cost(n);
        long long t = 0;
        double total = 0, max_tile = 0;
        for (int i = 0; i < n; i++) {
            begin[i] = t;
            tiles[i] = 1 + (long long)(rng() % ((rng() & 7) ? 8 : 200));
            cost[i] = (double)tiles[i] * (1.0 + (double)(rng() % 1000)) * (1.0 + (double)(rng() % 32));
            t += tiles[i];
            total += cost[i];
            max_tile = std::max(max_tile, cost[i] / (double)tiles[i]);
        }
        const int n_units = 1 + (int)(rng() % 20000);
        const auto p = rsgpu::plan_batch_units(begin, tiles, cost, n_units);
        if ((int)p.unit_first.size() != n_units + 1 || (int)p.unit_job.size() != n_units || p.unit_first[0] != 0 ||
            p.unit_first[n_units] != t) {
            std::printf("FAIL shape it=%d\n", it);
            return 1;
        }
        // cumulative cost at a tile boundary
        std::vector<double> tile_cost;
        tile_cost.reserve((size_t)t);
        for (int i = 0; i < n; i++)
            for (long long k = 0; k < tiles[i]; k++) tile_cost.push_back(cost[i] / (double)tiles[i]);
        std::vector<double> cum((size_t)t + 1, 0.0);
        for (long long x = 0; x < t; x++) cum[x + 1] = cum[x] + tile_cost[x];
        const double avg = total / n_units;
        for (int u = 0; u < n_units; u++) {
            const long long a = p.unit_first[u], b = p.unit_first[u + 1];
            if (b < a) {
                std::printf("FAIL order it=%d u=%d\n", it, u);
                return 1;
            }
            if (a < t) {
                const int j = p.unit_job[u];
                if (j < 0 || j >= n || begin[j] > a || a >= begin[j] + tiles[j]) {
                    std::printf("FAIL unit_job it=%d u=%d\n", it, u);
                    return 1;
                }
            }
            if (cum[b] - cum[a] > avg + max_tile + 1e-6 * total) {
                std::printf("FAIL balance it=%d u=%d cost=%g avg=%g tile=%g\n", it, u, cum[b] - cum[a], avg, max_tile);
                return 1;
            }
        }
    }
    std::printf("ok\n");
    return 0;
}
