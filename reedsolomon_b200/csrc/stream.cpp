// stream.cpp -- StreamEncoder (streaming.go:23-700) over host callbacks.
//
// The reference's rsStream reads one block (default 4 MiB) of every shard
// from io.Readers, runs the in-memory codec on the block and writes the
// produced shards to io.Writers, block after block.  Here the reads and
// writes are C callbacks run on the calling thread, and the device work of a
// block overlaps the callbacks of the next one: blocks alternate between two
// pinned host slots and two device slots; block b's H2D copy, contraction and
// D2H copy are queued on the context stream, then block b+1 is read while
// they run, and block b's outputs are written once its event completes.
//
// Block semantics follow readShards (streaming.go:255-288): every present
// reader is asked for a full block; a short read ends the stream and all
// short readers must agree on the size (ErrShardSize otherwise); a block of
// size 0 is the end of the stream (ErrShardNoData when it is the first).
#include <algorithm>
#include <cstring>

#include "rsgpu_internal.h"
#include "trace.h"

using namespace rsgpu;

namespace {

struct Slot {
    uint8_t *host = nullptr;   // total * block, pinned
    uint8_t *dev = nullptr;    // total * block
    int *h_flag = nullptr;     // pinned verify flag
    int *d_flag = nullptr;
    cudaEvent_t done = nullptr;
    size_t size = 0;           // bytes per shard in this block
    bool busy = false;
};

struct Pipeline {
    rsgpu_ctx *ctx;
    int total;
    size_t block;
    int extra;  // device-only rows per slot (recomputed parity for wide verifies)
    Slot slot[2];
    explicit Pipeline(rsgpu_ctx *c, int n, size_t b, int x = 0) : ctx(c), total(n), block(b), extra(x) {}
    int init() {
        for (Slot &s : slot) {
            RS_CUDA(cudaHostAlloc(&s.host, (size_t)total * block, cudaHostAllocPortable));
            RS_CUDA(cudaMalloc(&s.dev, (size_t)(total + extra) * block));
            RS_CUDA(cudaHostAlloc(&s.h_flag, sizeof(int), cudaHostAllocPortable));
            RS_CUDA(cudaMalloc(&s.d_flag, sizeof(int)));
            RS_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
        }
        return RS_OK;
    }
    ~Pipeline() {
        for (Slot &s : slot) {
            if (s.busy) cudaEventSynchronize(s.done);
            if (s.done) cudaEventDestroy(s.done);
            cudaFreeHost(s.host);
            cudaFree(s.dev);
            cudaFreeHost(s.h_flag);
            cudaFree(s.d_flag);
        }
    }
    uint8_t *h(Slot &s, int i) const { return s.host + (size_t)i * block; }
    uint8_t *d(Slot &s, int i) const { return s.dev + (size_t)i * block; }
};

// readShards: fills host rows of `want` shards; returns RS_OK with *size set,
// *eof when the block is empty.
int read_block(Pipeline &pl, Slot &s, const uint8_t *want, rsgpu_read_fn rd, void *user, size_t *size,
               bool *eof, int *err_shard) {
    long long short_size = -1;
    bool any_full = false;
    for (int i = 0; i < pl.total; i++) {
        if (!want[i]) continue;
        size_t got = 0;
        while (got < pl.block) {  // io.ReadFull
            const long long n = rd(user, i, pl.h(s, i) + got, pl.block - got);
            if (n < 0 || n > (long long)(pl.block - got)) {  // an error, or more than was asked for
                if (err_shard) *err_shard = i;
                return RS_ERR_STREAM_READ;
            }
            if (n == 0) break;
            got += (size_t)n;
        }
        if (got == pl.block) {
            any_full = true;
            continue;
        }
        if (short_size < 0) short_size = (long long)got;
        else if ((long long)got != short_size) return RS_ERR_SHARD_SIZE;
    }
    if (short_size == 0) {
        *eof = true;  // size 0 ends the stream (streaming.go:284-286)
        return RS_OK;
    }
    if (short_size > 0 && any_full) return RS_ERR_SHARD_SIZE;  // the codec rejects unequal shards
    *eof = false;
    *size = short_size < 0 ? pl.block : (size_t)short_size;
    return RS_OK;
}

int write_block(Pipeline &pl, Slot &s, const uint8_t *which, rsgpu_write_fn wr, void *user, int *err_shard) {
    for (int i = 0; i < pl.total; i++) {
        if (!which[i]) continue;
        if (wr(user, i, pl.h(s, i), s.size) != 0) {
            if (err_shard) *err_shard = i;
            return RS_ERR_STREAM_WRITE;
        }
    }
    return RS_OK;
}

bool classic_ok(rsgpu_encoder *enc) { return enc && enc->ctx && enc->codec == RS_CODEC_CLASSIC; }

}  // namespace

extern "C" {

int rsgpu_stream_encode(rsgpu_encoder *enc, rsgpu_read_fn rd, rsgpu_write_fn wr, void *user, size_t block,
                        int *err_shard) {
    RS_TRACE("rsgpu_stream_encode");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!classic_ok(enc)) return RS_ERR_NOT_SUPPORTED;  // rsStream wraps the classic codec
    if (!rd || !wr || block == 0) return RS_ERR_INVALID_INPUT;
    if (err_shard) *err_shard = -1;
    std::lock_guard<std::recursive_mutex> lk(enc->ctx->mu);
    const int k = enc->k, p = enc->p, total = enc->total;
    Pipeline pl(enc->ctx, total, block);
    int rc = pl.init();
    if (rc) return rc;
    std::vector<uint8_t> data(total, 0), parity(total, 0);
    for (int i = 0; i < k; i++) data[i] = 1;
    for (int i = k; i < total; i++) parity[i] = 1;
    std::vector<const uint8_t *> ins(k);
    std::vector<uint8_t *> outs(p);
    size_t read = 0;
    int prev = -1;
    for (int b = 0;; b++) {
        Slot &s = pl.slot[b & 1];
        if (s.busy) {  // block b-2 used this slot: its outputs were written when block b-1 was queued
            RS_CUDA(cudaEventSynchronize(s.done));
            s.busy = false;
        }
        bool eof = false;
        size_t size = 0;
        rc = read_block(pl, s, data.data(), rd, user, &size, &eof, err_shard);
        if (rc) return rc;
        if (eof) break;
        s.size = size;
        read += size;
        cudaStream_t st = enc->ctx->stream;
        for (int i = 0; i < k; i++) {
            RS_CUDA(cudaMemcpyAsync(pl.d(s, i), pl.h(s, i), size, cudaMemcpyHostToDevice, st));
            ins[i] = pl.d(s, i);
        }
        for (int o = 0; o < p; o++) outs[o] = pl.d(s, k + o);
        RS_CUDA(launch_gf8_matmul(st, enc->ctx->info, enc->parity_rows.data(), k, p, ins.data(), outs.data(), size,
                                  kModeWrite, enc->ctx->d_flag));
        for (int o = 0; o < p; o++)
            RS_CUDA(cudaMemcpyAsync(pl.h(s, k + o), pl.d(s, k + o), size, cudaMemcpyDeviceToHost, st));
        RS_CUDA(cudaEventRecord(s.done, st));
        s.busy = true;
        if (prev >= 0) {  // write the previous block while this one runs
            Slot &ps = pl.slot[prev];
            RS_CUDA(cudaEventSynchronize(ps.done));
            ps.busy = false;
            rc = write_block(pl, ps, parity.data(), wr, user, err_shard);
            if (rc) return rc;
        }
        prev = b & 1;
    }
    if (prev >= 0) {
        Slot &ps = pl.slot[prev];
        RS_CUDA(cudaEventSynchronize(ps.done));
        ps.busy = false;
        rc = write_block(pl, ps, parity.data(), wr, user, err_shard);
        if (rc) return rc;
    }
    return read == 0 ? RS_ERR_SHARD_NO_DATA : RS_OK;
}

int rsgpu_stream_verify(rsgpu_encoder *enc, rsgpu_read_fn rd, void *user, size_t block, int *ok, int *err_shard) {
    RS_TRACE("rsgpu_stream_verify");
    if (!enc || !ok) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!classic_ok(enc)) return RS_ERR_NOT_SUPPORTED;
    if (!rd || block == 0) return RS_ERR_INVALID_INPUT;
    if (err_shard) *err_shard = -1;
    *ok = 0;
    std::lock_guard<std::recursive_mutex> lk(enc->ctx->mu);
    const int k = enc->k, p = enc->p, total = enc->total;
    // more than kMaxIn inputs are tiled and accumulate, so the comparison
    // runs against parity recomputed into extra device rows
    const bool wide = k > kMaxIn;
    Pipeline pl(enc->ctx, total, block, wide ? p : 0);
    int rc = pl.init();
    if (rc) return rc;
    std::vector<uint8_t> all(total, 1);
    std::vector<const uint8_t *> ins(k), chk(p);
    size_t read = 0;
    int prev = -1;
    auto finished_ok = [&](Slot &s) -> int {
        RS_CUDA(cudaEventSynchronize(s.done));
        s.busy = false;
        return *s.h_flag == 0 ? 1 : 0;
    };
    for (int b = 0;; b++) {
        Slot &s = pl.slot[b & 1];
        if (s.busy && !finished_ok(s)) return RS_OK;  // a mismatch: *ok stays 0
        bool eof = false;
        size_t size = 0;
        rc = read_block(pl, s, all.data(), rd, user, &size, &eof, err_shard);
        if (rc) return rc;
        if (eof) break;
        s.size = size;
        read += size;
        cudaStream_t st = enc->ctx->stream;
        for (int i = 0; i < total; i++)
            RS_CUDA(cudaMemcpyAsync(pl.d(s, i), pl.h(s, i), size, cudaMemcpyHostToDevice, st));
        for (int i = 0; i < k; i++) ins[i] = pl.d(s, i);
        for (int o = 0; o < p; o++) chk[o] = pl.d(s, k + o);
        RS_CUDA(cudaMemsetAsync(s.d_flag, 0, sizeof(int), st));
        if (p > 0 && !wide) {
            RS_CUDA(launch_gf8_matmul(st, enc->ctx->info, enc->parity_rows.data(), k, p, ins.data(),
                                      const_cast<uint8_t *const *>(chk.data()), size, kModeVerify, s.d_flag));
        } else if (p > 0) {
            std::vector<uint8_t *> tmp(p);
            for (int o = 0; o < p; o++) tmp[o] = pl.d(s, total + o);
            RS_CUDA(launch_gf8_matmul(st, enc->ctx->info, enc->parity_rows.data(), k, p, ins.data(), tmp.data(),
                                      size, kModeWrite, s.d_flag));
            const uint8_t one = 1;
            for (int o = 0; o < p; o++) {
                const uint8_t *src = tmp[o];
                uint8_t *c = const_cast<uint8_t *>(chk[o]);
                RS_CUDA(launch_gf8_matmul(st, enc->ctx->info, &one, 1, 1, &src, &c, size, kModeVerify, s.d_flag));
            }
        }
        RS_CUDA(cudaMemcpyAsync(s.h_flag, s.d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        RS_CUDA(cudaEventRecord(s.done, st));
        s.busy = true;
        if (prev >= 0 && pl.slot[prev].busy && !finished_ok(pl.slot[prev])) return RS_OK;
        prev = b & 1;
    }
    for (Slot &s : pl.slot)
        if (s.busy && !finished_ok(s)) return RS_OK;
    if (read == 0) return RS_ERR_SHARD_NO_DATA;
    *ok = 1;
    return RS_OK;
}

int rsgpu_stream_reconstruct(rsgpu_encoder *enc, const uint8_t *valid, const uint8_t *fill, rsgpu_read_fn rd,
                             rsgpu_write_fn wr, void *user, size_t block, int *err_shard) {
    RS_TRACE("rsgpu_stream_reconstruct");
    if (!enc || !valid || !fill) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!classic_ok(enc)) return RS_ERR_NOT_SUPPORTED;
    if (!rd || !wr || block == 0) return RS_ERR_INVALID_INPUT;
    if (err_shard) *err_shard = -1;
    const int k = enc->k, total = enc->total;
    bool data_only = true;
    for (int i = 0; i < total; i++) {
        if (valid[i] && fill[i]) return RS_ERR_RECONSTRUCT_MISMATCH;
        if (i >= k && fill[i]) data_only = false;
    }
    std::lock_guard<std::recursive_mutex> lk(enc->ctx->mu);
    // The erasure pattern is the same for every block: plan it once
    // (reedsolomon.go:1670-1781 via Reconstruct / ReconstructData).
    std::vector<uint8_t> rows;
    std::vector<int> out_idx, in_idx;
    int rc = classic_decode_plan(enc, valid, data_only ? 1 : 0, nullptr, 0, rows, out_idx, in_idx);
    if (rc) return rc;
    Pipeline pl(enc->ctx, total, block);
    rc = pl.init();
    if (rc) return rc;
    std::vector<uint8_t> wants(fill, fill + total);
    for (int i = 0; i < total; i++) {  // fill writers of shards that need no rebuild get nothing
        bool rebuilt = std::find(out_idx.begin(), out_idx.end(), i) != out_idx.end();
        if (!rebuilt) wants[i] = 0;
    }
    std::vector<const uint8_t *> ins(in_idx.size());
    std::vector<uint8_t *> outs(out_idx.size());
    size_t read = 0;
    int prev = -1;
    for (int b = 0;; b++) {
        Slot &s = pl.slot[b & 1];
        if (s.busy) {
            RS_CUDA(cudaEventSynchronize(s.done));
            s.busy = false;
        }
        bool eof = false;
        size_t size = 0;
        rc = read_block(pl, s, valid, rd, user, &size, &eof, err_shard);
        if (rc) return rc;
        if (eof) break;
        s.size = size;
        read += size;
        cudaStream_t st = enc->ctx->stream;
        for (size_t j = 0; j < in_idx.size(); j++) {
            RS_CUDA(cudaMemcpyAsync(pl.d(s, in_idx[j]), pl.h(s, in_idx[j]), size, cudaMemcpyHostToDevice, st));
            ins[j] = pl.d(s, in_idx[j]);
        }
        for (size_t o = 0; o < out_idx.size(); o++) outs[o] = pl.d(s, out_idx[o]);
        if (!out_idx.empty())
            RS_CUDA(launch_gf8_matmul(st, enc->ctx->info, rows.data(), k, (int)out_idx.size(), ins.data(),
                                      outs.data(), size, kModeWrite, enc->ctx->d_flag));
        for (int i = 0; i < total; i++)
            if (wants[i]) RS_CUDA(cudaMemcpyAsync(pl.h(s, i), pl.d(s, i), size, cudaMemcpyDeviceToHost, st));
        RS_CUDA(cudaEventRecord(s.done, st));
        s.busy = true;
        if (prev >= 0) {
            Slot &ps = pl.slot[prev];
            RS_CUDA(cudaEventSynchronize(ps.done));
            ps.busy = false;
            rc = write_block(pl, ps, wants.data(), wr, user, err_shard);
            if (rc) return rc;
        }
        prev = b & 1;
    }
    if (prev >= 0) {
        Slot &ps = pl.slot[prev];
        RS_CUDA(cudaEventSynchronize(ps.done));
        ps.busy = false;
        rc = write_block(pl, ps, wants.data(), wr, user, err_shard);
        if (rc) return rc;
    }
    return read == 0 ? RS_ERR_SHARD_NO_DATA : RS_OK;
}

}  // extern "C"
