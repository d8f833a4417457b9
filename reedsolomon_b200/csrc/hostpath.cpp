// hostpath.cpp -- host-buffer entry points: PCIe copies inside the call.
//
// Every op on the hot path is column-local (classic RS bytewise, Leopard per
// 64-byte chunk), so the shards are processed in column chunks through a
// ring of device staging buffers: chunk c's H2D copies (copy_in stream) run
// while chunk c-1 is computed (context stream) and chunk c-2's results go
// back D2H (copy_out stream).  Events order the three streams per buffer.
#include <algorithm>
#include <cstring>

#include "rsgpu_internal.h"
#include "trace.h"

namespace rsgpu {
namespace {

constexpr int kRing = 3;

struct Pipeline {
    rsgpu_ctx *ctx;
    size_t chunk = 0;
    int rows = 0;  // staged rows per buffer
    cudaEvent_t in_done[kRing], comp_done[kRing], out_done[kRing];

    int init(int n_rows, size_t size, size_t align) {
        rows = n_rows;
        // ~8 chunks per call, at least 1 MiB per row, aligned for Leopard.
        size_t c = std::max<size_t>(size / 8, (size_t)1 << 20);
        c = std::min(c, size);
        c = (c + align - 1) / align * align;
        chunk = std::min(c, size);
        const size_t pitch = (chunk + 255) & ~(size_t)255;
        int rc = ctx->staging.ensure(pitch * (size_t)rows * kRing);
        if (rc) return rc;
        while (ctx->events.size() < 3 * kRing) {
            cudaEvent_t ev;
            RS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            ctx->events.push_back(ev);
        }
        for (int b = 0; b < kRing; b++) {
            in_done[b] = ctx->events[3 * b];
            comp_done[b] = ctx->events[3 * b + 1];
            out_done[b] = ctx->events[3 * b + 2];
        }
        return RS_OK;
    }
    uint8_t *row(int b, int r) const {
        const size_t pitch = (chunk + 255) & ~(size_t)255;
        return ctx->staging.ptr + pitch * ((size_t)b * rows + r);
    }
};

// Runs `compute(dev_rows, len)` over column chunks.  in_rows are copied
// host->device before compute, out_rows device->host after it.  Row r of a
// staging buffer corresponds to host_rows[r].
template <class F>
int run_pipeline(rsgpu_ctx *ctx, const std::vector<uint8_t *> &host_rows, const std::vector<int> &in_rows,
                 const std::vector<int> &out_rows, size_t size, size_t align, F compute) {
    Pipeline pl{ctx};
    int rc = pl.init((int)host_rows.size(), size, align);
    if (rc) return rc;
    std::vector<uint8_t *> dev(host_rows.size());
    int c = 0;
    for (size_t off = 0; off < size; off += pl.chunk, c++) {
        const size_t len = std::min(pl.chunk, size - off);
        const int b = c % kRing;
        if (c >= kRing) RS_CUDA(cudaStreamWaitEvent(ctx->copy_in, pl.out_done[b], 0));
        for (int r : in_rows)
            RS_CUDA(cudaMemcpyAsync(pl.row(b, r), host_rows[r] + off, len, cudaMemcpyHostToDevice, ctx->copy_in));
        RS_CUDA(cudaEventRecord(pl.in_done[b], ctx->copy_in));
        RS_CUDA(cudaStreamWaitEvent(ctx->stream, pl.in_done[b], 0));
        for (size_t r = 0; r < host_rows.size(); r++) dev[r] = pl.row(b, (int)r);
        rc = compute(dev, len);
        if (rc) return rc;
        RS_CUDA(cudaEventRecord(pl.comp_done[b], ctx->stream));
        RS_CUDA(cudaStreamWaitEvent(ctx->copy_out, pl.comp_done[b], 0));
        for (int r : out_rows)
            RS_CUDA(cudaMemcpyAsync(host_rows[r] + off, pl.row(b, r), len, cudaMemcpyDeviceToHost, ctx->copy_out));
        RS_CUDA(cudaEventRecord(pl.out_done[b], ctx->copy_out));
    }
    RS_CUDA(cudaStreamSynchronize(ctx->copy_out));
    RS_CUDA(cudaStreamSynchronize(ctx->stream));
    return RS_OK;
}

}  // namespace
}  // namespace rsgpu

using namespace rsgpu;

extern "C" int rsgpu_encode_host(rsgpu_encoder *enc, uint8_t *const *host, size_t size) {
    RS_TRACE("rsgpu_encode_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!host) return RS_ERR_TOO_FEW_SHARDS;
    for (int i = 0; i < enc->total; i++)
        if (!host[i]) return RS_ERR_SHARD_SIZE;
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    if (enc->p == 0) return RS_OK;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    std::vector<uint8_t *> rows(host, host + enc->total);
    std::vector<int> ins, outs;
    for (int i = 0; i < enc->k; i++) ins.push_back(i);
    for (int i = enc->k; i < enc->total; i++) outs.push_back(i);
    if (enc->codec != RS_CODEC_CLASSIC) {
        if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
        return run_pipeline(ctx, rows, ins, outs, size, 64, [&](std::vector<uint8_t *> &dev, size_t len) {
            return leo_encode_enqueue(enc, dev.data(), len);
        });
    }
    return run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, enc->parity_rows.data(), enc->k, enc->p,
                                  (const uint8_t *const *)dev.data(), dev.data() + enc->k, len,
                                  kModeWrite, ctx->d_flag));
        return RS_OK;
    });
}

extern "C" int rsgpu_reconstruct_host(rsgpu_encoder *enc, uint8_t **host, const uint8_t *present,
                                      size_t size, int data_only, uint8_t *written) {
    RS_TRACE("rsgpu_reconstruct_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!host || !present) return RS_ERR_TOO_FEW_SHARDS;
    if (written) memset(written, 0, (size_t)enc->total);
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (enc->codec != RS_CODEC_CLASSIC) {
        if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
        std::vector<int> ins, outs;
        int np = 0, dp = 0;
        for (int i = 0; i < enc->total; i++) {
            if (present[i]) {
                ins.push_back(i);
                np++;
                if (i < enc->k) dp++;
            } else if (i < enc->k || !data_only) {
                outs.push_back(i);
            }
        }
        if (np == 0) return RS_ERR_SHARD_NO_DATA;
        if (np == enc->total || (data_only && dp == enc->k)) return RS_OK;
        if (np < enc->k) return RS_ERR_TOO_FEW_SHARDS;
        for (int i : ins)
            if (!host[i]) return RS_ERR_SHARD_SIZE;
        for (int o : outs)
            if (!host[o]) return RS_ERR_INVALID_INPUT;  // host outputs must be preallocated
        std::vector<uint8_t *> rows(host, host + enc->total);
        int rc = run_pipeline(ctx, rows, ins, outs, size, 64, [&](std::vector<uint8_t *> &dev, size_t len) {
            return leo_reconstruct_enqueue(enc, dev.data(), present, len, !data_only);
        });
        if (rc == RS_OK && written)
            for (int o : outs) written[o] = 1;
        return rc;
    }
    std::vector<uint8_t> dec_rows;
    std::vector<int> out_idx, in_idx;
    int rc = classic_decode_plan(enc, present, data_only, nullptr, 0, dec_rows, out_idx, in_idx);
    if (rc || out_idx.empty()) return rc;
    for (int i : in_idx)
        if (!host[i]) return RS_ERR_SHARD_SIZE;
    for (int o : out_idx)
        if (!host[o]) return RS_ERR_INVALID_INPUT;
    // Stage only the k inputs and the outputs: rows [0,k) inputs, [k, k+n_out) outputs.
    std::vector<uint8_t *> rows;
    std::vector<int> ins, outs;
    for (size_t i = 0; i < in_idx.size(); i++) {
        rows.push_back(host[in_idx[i]]);
        ins.push_back((int)i);
    }
    for (size_t o = 0; o < out_idx.size(); o++) {
        rows.push_back(host[out_idx[o]]);
        outs.push_back((int)(in_idx.size() + o));
    }
    const int k = enc->k, n_out = (int)out_idx.size();
    rc = run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, dec_rows.data(), k, n_out,
                                  (const uint8_t *const *)dev.data(), dev.data() + k, len, kModeWrite,
                                  ctx->d_flag));
        return RS_OK;
    });
    if (rc == RS_OK && written)
        for (int o : out_idx) written[o] = 1;
    return rc;
}
