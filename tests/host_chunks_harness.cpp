// The host-buffer pipeline's column-chunk plan (reedsolomon_b200/csrc/
// host_chunks.h), checked on the CPU: exact plans for the documented cases,
// then random sizes, row counts, alignments and copy granularities, each
// plan covering [0, size) in order with every chunk at most the ring's row
// and every length but the last a multiple of the alignment (a Leopard call
// needs whole 64-byte columns in every chunk).
#include <cstdint>
#include <cstdio>
#include <random>

#include "host_chunks.h"

using rsgpu::plan_host_chunks;

static int fail(const char *what, size_t size, int rows, size_t align, double rpc) {
    std::printf("FAIL %s size=%zu rows=%d align=%zu rows_per_copy=%g\n", what, size, rows, align, rpc);
    return 1;
}

static bool same(const rsgpu::HostChunkPlan &p, const std::vector<size_t> &lens) {
    if (p.chunks.size() != lens.size()) return false;
    for (size_t i = 0; i < lens.size(); i++)
        if (p.chunks[i].second != lens[i]) return false;
    return true;
}

int main() {
    const size_t KiB = 1024, MiB = 1024 * KiB;
    // RS(10,4) x 64 MiB, 14 staged rows: shards in one block (10 and 4 rows
    // per copy) halve down to 256 KiB; one row per copy keeps 1 MiB chunks.
    if (!same(plan_host_chunks(64 * MiB, 14, 3, 16, 4.0),
              {16 * MiB, 16 * MiB, 16 * MiB, 8 * MiB, 4 * MiB, 2 * MiB, MiB, 512 * KiB, 256 * KiB, 256 * KiB}))
        return fail("64 MiB, 2D runs", 64 * MiB, 14, 16, 4.0);
    if (!same(plan_host_chunks(64 * MiB, 14, 3, 16, 1.0),
              {16 * MiB, 16 * MiB, 16 * MiB, 8 * MiB, 4 * MiB, 2 * MiB, MiB, MiB}))
        return fail("64 MiB, row copies", 64 * MiB, 14, 16, 1.0);
    if (!same(plan_host_chunks(MiB, 13, 3, 16, 4.0), {256 * KiB, 256 * KiB, 256 * KiB, 256 * KiB}))
        return fail("1 MiB, 2D runs of 4", MiB, 13, 16, 4.0);
    // RS(10,3) x 1 MiB in one block: 3 rows per copy out, minimum 1 MiB / 3
    // rounded up to 16 bytes
    if (!same(plan_host_chunks(MiB, 13, 3, 16, 3.0), {349536, 349536, 349504}))
        return fail("1 MiB, 2D runs of 3", MiB, 13, 16, 3.0);
    // 1.5 rows per copy: the minimum, 699050, rounds up to 699072 for Leopard
    if (plan_host_chunks(3 * MiB, 5, 3, 64, 1.5).min_chunk != 699072)
        return fail("minimum rounded to the alignment", 3 * MiB, 5, 64, 1.5);
    if (!same(plan_host_chunks(MiB, 13, 3, 16, 1.0), {MiB})) return fail("1 MiB, row copies", MiB, 13, 16, 1.0);
    std::mt19937_64 rng(12345);
    const double rpcs[] = {1.0, 1.5, 2.0, 3.0, 4.0, 7.0, 10.0, 1e9};
    for (int it = 0; it < 200000; it++) {
        const size_t align = (rng() & 1) ? 64 : 16;
        size_t size = 1 + rng() % (300 * MiB);
        if (align == 64) size = std::max<size_t>(64, size / 64 * 64);
        const int rows = 2 + (int)(rng() % 3000);
        const double rpc = rpcs[rng() % 8];
        const auto p = plan_host_chunks(size, rows, 3, align, rpc);
        size_t off = 0;
        for (size_t i = 0; i < p.chunks.size(); i++) {
            const auto &c = p.chunks[i];
            if (c.first != off || c.second == 0 || c.second > p.chunk) return fail("coverage", size, rows, align, rpc);
            if (i + 1 < p.chunks.size() && c.second % align) return fail("alignment", size, rows, align, rpc);
            off += c.second;
        }
        if (off != size) return fail("total", size, rows, align, rpc);
        if (p.chunks.size() > 20000) return fail("count", size, rows, align, rpc);
    }
    std::printf("ok\n");
    return 0;
}
