// rsgpu_internal.h -- context / encoder state shared by the runtime sources.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/rsgpu.h"
#include "gf_host.h"
#include "kernels.h"

namespace rsgpu {

void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

#define RS_CUDA(call)                                     \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) return cuda_status(_e, #call); \
    } while (0)

struct LeoState;        // leopard.cu
struct LeoErrLocCache;  // leopard.cu

// Grow-only device buffer owned by a context.
struct DeviceBuffer {
    uint8_t *ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
};

}  // namespace rsgpu

struct rsgpu_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;  // host-path copy streams
    rsgpu::DeviceInfo info;
    int *d_flag = nullptr;
    int *h_flag = nullptr;  // pinned
    std::recursive_mutex mu;
    rsgpu::DeviceBuffer scratch;  // verify temporaries, leopard work rows
    rsgpu::DeviceBuffer staging;  // host-path device copies of shards
    std::vector<cudaEvent_t> events;
    // Host row layouts (first row, stride, rows) whose 2D copy the driver
    // rejected (rows of separate allocations): copied row by row from then on.
    std::vector<std::tuple<const uint8_t *, size_t, int>> rejected_2d;
    std::shared_ptr<rsgpu::LeoState> leo;  // Leopard tables, built on first use
    cudaMemPool_t pool = nullptr;  // stream-ordered scratch (keeps its memory, never trims)
};

struct rsgpu_encoder {
    rsgpu_ctx *ctx = nullptr;
    int k = 0, p = 0, total = 0;
    int codec = RS_CODEC_CLASSIC;
    rsgpu_options opts{};
    rsgpu::Matrix m;                      // (k+p) x k classic encoding matrix
    std::vector<uint8_t> parity_rows;     // p x k
    std::unique_ptr<rsgpu::InversionTree> tree;
    std::shared_ptr<rsgpu::LeoState> leo;
    std::shared_ptr<rsgpu::LeoErrLocCache> errlocs;  // Leopard error locators per erasure pattern
};

namespace rsgpu {
// Classic codec helpers (encoder.cpp)
int classic_decode_plan(rsgpu_encoder *enc, const uint8_t *present, int data_only,
                        const uint8_t *required, int n_required, std::vector<uint8_t> &rows,
                        std::vector<int> &out_idx, std::vector<int> &in_idx);
int decode_idx_plan(rsgpu_encoder *enc, const uint8_t *expect, const uint8_t *has_in, const uint8_t *has_dst,
                    std::vector<uint8_t> &rows, std::vector<int> &in_shards, std::vector<int> &out_shards);
// Leopard codec (leopard.cu)
int leo_create(rsgpu_encoder *enc);
int leo_encode(rsgpu_encoder *enc, uint8_t *const *shards, size_t size);
int leo_verify(rsgpu_encoder *enc, uint8_t *const *shards, size_t size, int *ok);
int leo_reconstruct(rsgpu_encoder *enc, uint8_t **shards, const uint8_t *present, size_t size,
                    int recover_all, uint8_t *written);
int leo_errloc_cached(const rsgpu_encoder *enc);  // cached erasure patterns
// Enqueue-only variants on the context stream (no host synchronisation);
// all shard pointers must be valid device buffers of `size` bytes.
int leo_encode_enqueue(rsgpu_encoder *enc, uint8_t *const *shards, size_t size, cudaStream_t st = nullptr);
int leo_reconstruct_enqueue(rsgpu_encoder *enc, uint8_t *const *shards, const uint8_t *present,
                            size_t size, int recover_all, cudaStream_t st = nullptr);
// Batched execution on an explicit stream (batch.cu).
int batch_run_on(rsgpu_batch *b, int mode, cudaStream_t st);
int batch_stripe_count(const rsgpu_batch *b);
// Copies the verify outcomes of a finished run (stream-ordered on st).
int batch_read_flags(rsgpu_batch *b, int *ok, int n, cudaStream_t st);
}  // namespace rsgpu
