// host_chunks.h -- column-chunk plan of the host-buffer pipeline (hostpath.cpp).
//
// Pure host code (no CUDA), so the plan's invariants are tested on the CPU
// (tests/host_chunks_harness.cpp): the chunks cover [0, size) in order, none
// is longer than the staging ring's row, and every length but the last is
// a multiple of the codec's alignment (Leopard works on whole 64-byte
// columns).
#pragma once

#include <algorithm>
#include <cstddef>
#include <utility>
#include <vector>

namespace rsgpu {

// Smallest column chunk per row: 256 KiB when the rows move as 2D runs (a
// 1 MiB shard still splits into four, so its copies in, compute and copies
// out overlap), up to 1 MiB when they move one row per copy (a copy's fixed
// cost, a few microseconds, must stay small against its bytes).
constexpr size_t kHostMinChunk = (size_t)256 << 10;
constexpr size_t kHostMinCopyBytes = (size_t)1 << 20;
constexpr size_t kHostRingBytes = (size_t)1 << 30;  // staging ring cap (wide Leopard stripes)

struct HostChunkPlan {
    size_t chunk = 0;      // largest chunk: the staging ring's row size
    size_t min_chunk = 0;  // the tail halves down to this
    std::vector<std::pair<size_t, size_t>> chunks;  // (offset, length)
};

// size bytes per row, rows staged per ring buffer, ring buffers, the
// codec's alignment, and the fewest rows one copy moves on average in
// either direction (1 for row-by-row copies).  About four full chunks per
// call, then halves down to min_chunk, so the last chunk, whose compute and
// copies out nothing overlaps, is small.
inline HostChunkPlan plan_host_chunks(size_t size, int rows, int ring, size_t align, double rows_per_copy) {
    HostChunkPlan p;
    if (size == 0) return p;
    p.min_chunk = std::min(kHostMinCopyBytes,
                           std::max(kHostMinChunk, (size_t)((double)kHostMinCopyBytes / std::max(1.0, rows_per_copy))));
    p.min_chunk = (p.min_chunk + align - 1) / align * align;
    size_t c = std::max<size_t>(size / 4, p.min_chunk);
    const size_t budget = kHostRingBytes / ((size_t)std::max(1, rows) * (size_t)std::max(1, ring));
    c = std::min(c, std::max(budget, align));
    c = std::min(c, size);
    c = (c + align - 1) / align * align;
    p.chunk = std::min(c, size);
    const size_t tail_min = std::max<size_t>(p.min_chunk, align);
    size_t off = 0;
    while (off < size) {
        const size_t rem = size - off;
        size_t len = p.chunk;
        if (rem < 2 * p.chunk) {
            len = rem <= tail_min ? rem : std::max(tail_min, (rem / 2 + align - 1) / align * align);
            len = std::min(len, std::min(p.chunk, rem));
        }
        p.chunks.emplace_back(off, len);
        off += len;
    }
    return p;
}

}  // namespace rsgpu
