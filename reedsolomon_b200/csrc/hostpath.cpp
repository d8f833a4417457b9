// hostpath.cpp -- host-buffer entry points: PCIe copies inside the call.
//
// Every op on the hot path is column-local (classic RS bytewise, Leopard per
// 64-byte chunk), so the shards are processed in column chunks through a
// ring of device staging buffers: chunk c's H2D copies (copy_in stream) run
// while chunk c-1 is computed (context stream) and chunk c-2's results go
// back D2H (copy_out stream).  Events order the three streams per buffer.
#include <algorithm>
#include <cstring>

#include "host_chunks.h"
#include "rsgpu_internal.h"
#include "trace.h"

namespace rsgpu {
namespace {

constexpr int kRing = 3;

struct Pipeline {
    rsgpu_ctx *ctx;
    size_t chunk = 0;  // largest column chunk (the staging ring's row size)
    int rows = 0;      // staged rows per buffer
    cudaEvent_t in_done[kRing], comp_done[kRing], out_done[kRing];
    HostChunkPlan plan;

    // rows_per_copy: the fewest rows one copy moves on average, in either
    // direction (1 for row-by-row copies); the chunks: host_chunks.h.
    int init(int n_rows, size_t size, size_t align, double rows_per_copy) {
        rows = n_rows;
        plan = plan_host_chunks(size, rows, kRing, align, rows_per_copy);
        chunk = plan.chunk;
        int rc = ctx->staging.ensure(pitch() * (size_t)rows * kRing);
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
    size_t pitch() const { return (chunk + 255) & ~(size_t)255; }
    uint8_t *row(int b, int r) const { return ctx->staging.ptr + pitch() * ((size_t)b * rows + r); }
};

// Rows of one copy direction, as runs: consecutive staging rows (indices)
// that sit at one stride in host memory (the layout of Split's shards or of
// one allocation cut into shards, unsafe.go:19-43) move with one 2D copy per
// chunk; a run of one row (stride 0) with a plain copy.  A constant stride
// between separate allocations is possible too; the driver rejects a 2D copy
// whose span crosses them (invalid value) or whose stride exceeds its
// largest pitch (invalid pitch), and that run is then copied row by row.
struct Run {
    int first, count;  // staging rows first .. first+count-1
    size_t stride;     // host bytes between them, 0: one row at a time
};

bool rejected(const rsgpu_ctx *ctx, const uint8_t *first, size_t stride, int count) {
    for (const auto &t : ctx->rejected_2d)
        if (std::get<0>(t) == first && std::get<1>(t) == stride && std::get<2>(t) == count) return true;
    return false;
}

std::vector<Run> make_runs(const rsgpu_ctx *ctx, const std::vector<uint8_t *> &host_rows,
                           const std::vector<int> &idx, size_t size) {
    std::vector<Run> runs;
    for (size_t j = 0; j < idx.size();) {
        Run r{idx[j], 1, 0};
        if (j + 1 < idx.size() && idx[j + 1] == idx[j] + 1) {
            const ptrdiff_t st = host_rows[idx[j + 1]] - host_rows[idx[j]];
            if (st > 0 && (size_t)st >= size) {
                r.stride = (size_t)st;
                while (j + r.count < idx.size() && idx[j + r.count] == idx[j] + r.count &&
                       host_rows[idx[j + r.count]] - host_rows[idx[j + r.count - 1]] == st)
                    r.count++;
                if (rejected(ctx, host_rows[r.first], r.stride, r.count)) {
                    for (int q = 0; q < r.count; q++) runs.push_back(Run{r.first + q, 1, 0});
                    j += r.count;
                    continue;
                }
            }
        }
        runs.push_back(r);
        j += r.count;
    }
    return runs;
}

// Copies column [off, off + len) of every row of the runs, host to staging
// buffer b (h2d) or back, on stream st.
int copy_runs(const Pipeline &pl, std::vector<Run> &runs, const std::vector<uint8_t *> &host_rows, int b,
              size_t off, size_t len, bool h2d, cudaStream_t st) {
    rsgpu_ctx *ctx = pl.ctx;
    for (Run &r : runs) {
        if (r.stride) {
            cudaError_t e =
                h2d ? cudaMemcpy2DAsync(pl.row(b, r.first), pl.pitch(), host_rows[r.first] + off, r.stride, len,
                                        r.count, cudaMemcpyHostToDevice, st)
                    : cudaMemcpy2DAsync(host_rows[r.first] + off, r.stride, pl.row(b, r.first), pl.pitch(), len,
                                        r.count, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) continue;
            // a span across allocations (invalid value) or a stride past the
            // largest pitch a copy takes (invalid pitch): row copies from now on
            if (e != cudaErrorInvalidValue && e != cudaErrorInvalidPitchValue) RS_CUDA(e);
            cudaGetLastError();
            if (ctx->rejected_2d.size() >= 64) ctx->rejected_2d.erase(ctx->rejected_2d.begin());
            ctx->rejected_2d.emplace_back(host_rows[r.first], r.stride, r.count);
            r.stride = 0;
        }
        for (int q = r.first; q < r.first + r.count; q++) {
            if (h2d) RS_CUDA(cudaMemcpyAsync(pl.row(b, q), host_rows[q] + off, len, cudaMemcpyHostToDevice, st));
            else RS_CUDA(cudaMemcpyAsync(host_rows[q] + off, pl.row(b, q), len, cudaMemcpyDeviceToHost, st));
        }
    }
    return RS_OK;
}

// Runs `compute(dev_rows, len)` over column chunks.  in_rows are copied
// host->device before compute, out_rows device->host after it.  Row r of a
// staging buffer corresponds to host_rows[r].
template <class F>
int run_pipeline(rsgpu_ctx *ctx, const std::vector<uint8_t *> &host_rows, const std::vector<int> &in_rows,
                 const std::vector<int> &out_rows, size_t size, size_t align, F compute) {
    std::vector<Run> in_runs = make_runs(ctx, host_rows, in_rows, size),
                     out_runs = make_runs(ctx, host_rows, out_rows, size);
    auto per_copy = [](const std::vector<int> &idx, const std::vector<Run> &runs) {
        return runs.empty() ? 1e9 : (double)idx.size() / (double)runs.size();
    };
    Pipeline pl{ctx};
    int rc = pl.init((int)host_rows.size(), size, align,
                     std::min(per_copy(in_rows, in_runs), per_copy(out_rows, out_runs)));
    if (rc) return rc;
    std::vector<uint8_t *> dev(host_rows.size());
    int c = 0;
    for (const auto &ch : pl.plan.chunks) {
        const size_t off = ch.first, len = ch.second;
        const int b = c % kRing;
        if (c >= kRing) RS_CUDA(cudaStreamWaitEvent(ctx->copy_in, pl.out_done[b], 0));
        rc = copy_runs(pl, in_runs, host_rows, b, off, len, true, ctx->copy_in);
        if (rc) return rc;
        RS_CUDA(cudaEventRecord(pl.in_done[b], ctx->copy_in));
        RS_CUDA(cudaStreamWaitEvent(ctx->stream, pl.in_done[b], 0));
        for (size_t r = 0; r < host_rows.size(); r++) dev[r] = pl.row(b, (int)r);
        rc = compute(dev, len);
        if (rc) return rc;
        RS_CUDA(cudaEventRecord(pl.comp_done[b], ctx->stream));
        RS_CUDA(cudaStreamWaitEvent(ctx->copy_out, pl.comp_done[b], 0));
        rc = copy_runs(pl, out_runs, host_rows, b, off, len, false, ctx->copy_out);
        if (rc) return rc;
        RS_CUDA(cudaEventRecord(pl.out_done[b], ctx->copy_out));
        c++;
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

namespace {

// Host-buffer Reconstruct / ReconstructData / ReconstructSome: the inputs
// (the first k present shards, classic; every present shard, Leopard) go
// H2D, the rebuilt shards D2H, per column chunk.  Host outputs must be
// preallocated.
int reconstruct_host_common(rsgpu_encoder *enc, uint8_t **host, const uint8_t *present, size_t size, int data_only,
                            const uint8_t *required, int n_required, uint8_t *written) {
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (!host || !present) return RS_ERR_TOO_FEW_SHARDS;
    if (written) memset(written, 0, (size_t)enc->total);
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (enc->codec != RS_CODEC_CLASSIC) {
        if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
        // leopard.go:378-391: ReconstructSome recovers parity only when
        // required covers every shard; it is otherwise data-only.
        if (required) data_only = n_required != enc->total;
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
    int rc = classic_decode_plan(enc, present, data_only, required, n_required, dec_rows, out_idx, in_idx);
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

}  // namespace

extern "C" int rsgpu_reconstruct_host(rsgpu_encoder *enc, uint8_t **host, const uint8_t *present,
                                      size_t size, int data_only, uint8_t *written) {
    RS_TRACE("rsgpu_reconstruct_host");
    return reconstruct_host_common(enc, host, present, size, data_only, nullptr, 0, written);
}

extern "C" int rsgpu_reconstruct_some_host(rsgpu_encoder *enc, uint8_t **host, const uint8_t *present,
                                           const uint8_t *required, int n_required, size_t size,
                                           uint8_t *written) {
    RS_TRACE("rsgpu_reconstruct_some_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    // reedsolomon.go:1655-1660
    if (!required || (n_required != enc->k && n_required != enc->total)) return RS_ERR_INVALID_INPUT;
    return reconstruct_host_common(enc, host, present, size, n_required == enc->k, required, n_required,
                                   written);
}

extern "C" int rsgpu_verify_host(rsgpu_encoder *enc, uint8_t *const *host, size_t size, int *ok) {
    RS_TRACE("rsgpu_verify_host");
    if (!enc || !ok) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    *ok = 0;
    if (!host) return RS_ERR_TOO_FEW_SHARDS;
    for (int i = 0; i < enc->total; i++)
        if (!host[i]) return RS_ERR_SHARD_SIZE;
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    if (enc->p == 0) {
        *ok = 1;
        return RS_OK;
    }
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    const int k = enc->k, p = enc->p, total = enc->total;
    // every shard goes H2D; nothing comes back but the mismatch flag
    std::vector<uint8_t *> rows(host, host + total);
    std::vector<int> ins, outs;
    for (int i = 0; i < total; i++) ins.push_back(i);
    RS_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
    int rc;
    if (enc->codec != RS_CODEC_CLASSIC) {
        if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
        // Leopard (leopard.go:393-419): re-encode into p staging rows past the
        // shards (never copied), then compare them with the received parity.
        for (int i = 0; i < p; i++) rows.push_back(nullptr);
        rc = run_pipeline(ctx, rows, ins, outs, size, 64, [&](std::vector<uint8_t *> &dev, size_t len) {
            std::vector<uint8_t *> tmp(dev.begin(), dev.begin() + total);
            for (int i = 0; i < p; i++) tmp[k + i] = dev[total + i];
            int r = leo_encode_enqueue(enc, tmp.data(), len);
            if (r) return r;
            const uint8_t one = 1;
            for (int i = 0; i < p; i++) {
                const uint8_t *src = dev[total + i];
                RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, &one, 1, 1, &src, &dev[k + i], len, kModeVerify,
                                          ctx->d_flag));
            }
            return RS_OK;
        });
    } else {
        // reedsolomon.go:857-871 with checkSomeShards fused: parity compared in place
        rc = run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
            RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, enc->parity_rows.data(), k, p,
                                      (const uint8_t *const *)dev.data(), dev.data() + k, len, kModeVerify,
                                      ctx->d_flag));
            return RS_OK;
        });
    }
    if (rc) return rc;
    RS_CUDA(cudaMemcpyAsync(ctx->h_flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RS_CUDA(cudaStreamSynchronize(ctx->stream));
    *ok = (*ctx->h_flag == 0);
    return RS_OK;
}

extern "C" int rsgpu_encode_idx_host(rsgpu_encoder *enc, const uint8_t *host_data, int idx, uint8_t *const *host_parity,
                                     size_t size) {
    RS_TRACE("rsgpu_encode_idx_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (enc->codec != RS_CODEC_CLASSIC) return RS_ERR_NOT_SUPPORTED;  // leopard.go:272
    if (enc->p == 0) return RS_OK;
    if (idx < 0 || idx >= enc->k) return RS_ERR_INV_SHARD_NUM;
    if (!host_parity) return RS_ERR_TOO_FEW_SHARDS;
    for (int o = 0; o < enc->p; o++)
        if (!host_parity[o]) return RS_ERR_SHARD_SIZE;
    if (!host_data) return RS_ERR_SHARD_SIZE;
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    const int p = enc->p;
    // parity[o] ^= M[k+o][idx] * data (reedsolomon.go:708-757): the data and
    // the parity go H2D, the parity comes back
    std::vector<uint8_t> col(p);
    for (int o = 0; o < p; o++) col[o] = enc->parity_rows[(size_t)o * enc->k + idx];
    std::vector<uint8_t *> rows{const_cast<uint8_t *>(host_data)};
    std::vector<int> ins{0}, outs;
    for (int o = 0; o < p; o++) {
        rows.push_back(host_parity[o]);
        ins.push_back(1 + o);
        outs.push_back(1 + o);
    }
    return run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, col.data(), 1, p, (const uint8_t *const *)dev.data(),
                                  dev.data() + 1, len, kModeXor, ctx->d_flag));
        return RS_OK;
    });
}

extern "C" int rsgpu_update_host(rsgpu_encoder *enc, uint8_t *const *host, const uint8_t *const *host_new,
                                 size_t size) {
    RS_TRACE("rsgpu_update_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (enc->codec != RS_CODEC_CLASSIC) return RS_ERR_NOT_SUPPORTED;  // leopard.go:316, leopard8.go:289
    if (!host || !host_new) return RS_ERR_TOO_FEW_SHARDS;
    if (size == 0) return RS_ERR_SHARD_NO_DATA;
    const int k = enc->k, p = enc->p;
    std::vector<int> cols;
    for (int c = 0; c < k; c++)
        if (host_new[c]) {
            if (!host[c]) return RS_ERR_INVALID_INPUT;
            cols.push_back(c);
        }
    if (cols.empty()) return RS_ERR_SHARD_NO_DATA;  // checkShards(newDatashards, true)
    for (int o = 0; o < p; o++)
        if (!host[k + o]) return RS_ERR_INVALID_INPUT;
    if (p == 0) return RS_OK;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    // reedsolomon.go:762-853: rows [0,n) the changed shards (left holding the
    // delta, like the reference), [n,2n) their new data, [2n,2n+p) parity
    const int n = (int)cols.size();
    std::vector<uint8_t> prow((size_t)p * n);
    std::vector<uint8_t *> rows;
    std::vector<int> ins, outs;
    for (int j = 0; j < n; j++) {
        rows.push_back(host[cols[j]]);
        ins.push_back(j);
        outs.push_back(j);
        for (int o = 0; o < p; o++) prow[(size_t)o * n + j] = enc->parity_rows[(size_t)o * k + cols[j]];
    }
    for (int j = 0; j < n; j++) {
        rows.push_back(const_cast<uint8_t *>(host_new[cols[j]]));
        ins.push_back(n + j);
    }
    for (int o = 0; o < p; o++) {
        rows.push_back(host[k + o]);
        ins.push_back(2 * n + o);
        outs.push_back(2 * n + o);
    }
    return run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
        for (int j = 0; j < n; j++) RS_CUDA(launch_xor(ctx->stream, ctx->info, dev[n + j], dev[j], len));
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, prow.data(), n, p, (const uint8_t *const *)dev.data(),
                                  dev.data() + 2 * n, len, kModeXor, ctx->d_flag));
        return RS_OK;
    });
}

extern "C" int rsgpu_decode_idx_host(rsgpu_encoder *enc, uint8_t *const *host_dst, const uint8_t *expect,
                                     const uint8_t *const *host_input, size_t size) {
    RS_TRACE("rsgpu_decode_idx_host");
    if (!enc) return RS_ERR_INVALID_INPUT;
    if (!enc->ctx) return RS_ERR_NO_DEVICE;
    if (enc->codec != RS_CODEC_CLASSIC) return RS_ERR_NOT_SUPPORTED;  // leopard.go:94, leopard8.go:90
    if (!host_dst || !host_input) return RS_ERR_INVALID_INPUT;
    rsgpu_ctx *ctx = enc->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    const int total = enc->total;
    std::vector<uint8_t *> rows;
    std::vector<int> ins, outs;
    if (!expect) {  // merging mode: dst[i] ^= input[i]
        for (int i = 0; i < total; i++)
            if (host_input[i] && !host_dst[i]) return RS_ERR_INVALID_INPUT;
        if (size == 0) return RS_OK;
        std::vector<int> pairs;
        for (int i = 0; i < total; i++)
            if (host_input[i]) pairs.push_back(i);
        if (pairs.empty()) return RS_OK;
        const int n = (int)pairs.size();
        for (int j = 0; j < n; j++) {
            rows.push_back(const_cast<uint8_t *>(host_input[pairs[j]]));
            ins.push_back(j);
        }
        for (int j = 0; j < n; j++) {
            rows.push_back(host_dst[pairs[j]]);
            ins.push_back(n + j);
            outs.push_back(n + j);
        }
        return run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
            for (int j = 0; j < n; j++) RS_CUDA(launch_xor(ctx->stream, ctx->info, dev[j], dev[n + j], len));
            return RS_OK;
        });
    }
    std::vector<uint8_t> has_in(total), has_dst(total);
    for (int i = 0; i < total; i++) {
        has_in[i] = host_input[i] != nullptr;
        has_dst[i] = host_dst[i] != nullptr;
    }
    std::vector<uint8_t> dec_rows;
    std::vector<int> in_sh, out_sh;
    int rc = decode_idx_plan(enc, expect, has_in.data(), has_dst.data(), dec_rows, in_sh, out_sh);
    if (rc || in_sh.empty() || out_sh.empty() || size == 0) return rc;
    const int n_in = (int)in_sh.size(), n_out = (int)out_sh.size();
    for (int j = 0; j < n_in; j++) {
        rows.push_back(const_cast<uint8_t *>(host_input[in_sh[j]]));
        ins.push_back(j);
    }
    for (int o = 0; o < n_out; o++) {  // accumulated: read, updated, written back
        rows.push_back(host_dst[out_sh[o]]);
        ins.push_back(n_in + o);
        outs.push_back(n_in + o);
    }
    return run_pipeline(ctx, rows, ins, outs, size, 16, [&](std::vector<uint8_t *> &dev, size_t len) {
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, dec_rows.data(), n_in, n_out,
                                  (const uint8_t *const *)dev.data(), dev.data() + n_in, len, kModeXor,
                                  ctx->d_flag));
        return RS_OK;
    });
}
