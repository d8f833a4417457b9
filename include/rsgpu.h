/*
 * rsgpu.h -- C-ABI of the B200 erasure-coding engine (librsgpu.so).
 *
 * Drop-in boundary for klauspost/reedsolomon's hot path.  Each entry point
 * names the reference interface it replaces (paths inside the reference
 * project).  All functions are plain C: pointers and sizes only.
 *
 * Memory model
 *   - "shards" arguments of the device entry points are host arrays of DEVICE
 *     pointers (one per shard), like the reference's [][]byte.
 *   - *_host entry points take host arrays of HOST pointers; the library moves
 *     the bytes over PCIe (pinned host memory gives full PCIe bandwidth).
 *   - The caller owns every shard buffer.  A missing output shard passed as
 *     NULL is allocated by the library (rsgpu_free releases it), mirroring the
 *     reference's AllocAligned of missing shards (reedsolomon.go:1747-1751).
 *   - A missing shard is marked by present[i] == 0 (the reference uses a
 *     zero-length slice, reedsolomon.go:1680-1696).
 *   - Calls are synchronous with respect to the host unless named *_async:
 *     they enqueue on the context stream and wait, keeping the reference's
 *     blocking semantics.
 *
 * Status codes map 1:1 onto the reference's sentinel errors.
 */
#ifndef RSGPU_H
#define RSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define RS_OK 0
#define RS_ERR_TOO_FEW_SHARDS -1        /* ErrTooFewShards      reedsolomon.go:678 */
#define RS_ERR_SHARD_NO_DATA -2         /* ErrShardNoData       reedsolomon.go:1391 */
#define RS_ERR_SHARD_SIZE -3            /* ErrShardSize         reedsolomon.go:1395 */
#define RS_ERR_INVALID_SHARD_SIZE -4    /* ErrInvalidShardSize  reedsolomon.go:1399 */
#define RS_ERR_INV_SHARD_NUM -5         /* ErrInvShardNum       reedsolomon.go:216 */
#define RS_ERR_MAX_SHARD_NUM -6         /* ErrMaxShardNum       reedsolomon.go:221 */
#define RS_ERR_NOT_SUPPORTED -7         /* ErrNotSupported      reedsolomon.go:224 */
#define RS_ERR_INVALID_INPUT -8         /* ErrInvalidInput      reedsolomon.go:760 */
#define RS_ERR_RECONSTRUCT_REQUIRED -9  /* ErrReconstructRequired reedsolomon.go:1862 */
#define RS_ERR_SINGULAR -10             /* errSingular          matrix.go:184 */
#define RS_ERR_NOT_SQUARE -11           /* errNotSquare         matrix.go:187 */
#define RS_ERR_SHORT_DATA -12           /* ErrShortData         reedsolomon.go:1785 */
#define RS_ERR_RECONSTRUCT_MISMATCH -13 /* ErrReconstructMismatch streaming.go:457 */
#define RS_ERR_STREAM_READ -14          /* StreamReadError      streaming.go:93-109 */
#define RS_ERR_STREAM_WRITE -15         /* StreamWriteError     streaming.go:111-127 */
#define RS_ERR_CUDA -100                /* a CUDA call failed (see rsgpu_last_error) */
#define RS_ERR_NOMEM -101               /* device or pinned allocation failed */
#define RS_ERR_TIMEOUT -102             /* a bounded device wait expired */
#define RS_ERR_NO_DEVICE -103           /* encoder has no device context */

/* ---- codecs and matrix kinds --------------------------------------------- */
#define RS_CODEC_CLASSIC 0   /* reedSolomon (reedsolomon.go:170) */
#define RS_CODEC_LEOPARD16 1 /* leopardFF16 (leopard.go:36) */
#define RS_CODEC_LEOPARD8 2  /* leopardFF8  (leopard8.go:22) */

#define RS_MATRIX_DEFAULT 0  /* buildMatrix          reedsolomon.go:232 */
#define RS_MATRIX_CAUCHY 1   /* WithCauchyMatrix     options.go:249 */
#define RS_MATRIX_PAR1 2     /* WithPAR1Matrix       options.go:237 */
#define RS_MATRIX_JERASURE 3 /* WithJerasureMatrix   options.go:225 */

#define RS_LEOPARD_AS_NEEDED 0 /* leopardAsNeeded options.go:68 */
#define RS_LEOPARD_GF16 1      /* WithLeopardGF16 options.go:283 */
#define RS_LEOPARD_ALWAYS 2    /* WithLeopardGF   options.go:297 */

typedef struct rsgpu_ctx rsgpu_ctx;
typedef struct rsgpu_encoder rsgpu_encoder;

/* Functional options of New (options.go:13-44).  CPU-tuning options
 * (goroutines, split sizes, ISA toggles, stream options) have no meaning on
 * the GPU and are absent. */
typedef struct rsgpu_options {
    int matrix_kind;             /* RS_MATRIX_*; options.go:225-258 */
    int fast_one_parity;         /* WithFastOneParityMatrix options.go:260 */
    int leopard;                 /* RS_LEOPARD_*; WithLeopardGF16 / WithLeopardGF */
    int inversion_cache;         /* WithInversionCache options.go:152 (default 1) */
    const uint8_t *custom_matrix;/* WithCustomMatrix options.go:272: rows x cols, row-major, or NULL */
    int custom_rows, custom_cols;
} rsgpu_options;

/* ---- context: device, stream, scratch ------------------------------------ */
/* Creates a context on `device` with its own non-blocking stream. */
int rsgpu_ctx_create(int device, rsgpu_ctx **out);
int rsgpu_ctx_destroy(rsgpu_ctx *ctx);
/* Run on an external cudaStream_t, used verbatim (NULL is the legacy default
 * stream); rsgpu_ctx_reset_stream returns to the context's own stream. */
int rsgpu_ctx_set_stream(rsgpu_ctx *ctx, void *cuda_stream);
int rsgpu_ctx_reset_stream(rsgpu_ctx *ctx);
void *rsgpu_ctx_stream(rsgpu_ctx *ctx);
int rsgpu_ctx_synchronize(rsgpu_ctx *ctx);
/* Human-readable name of a status code, and the last error text of this thread. */
const char *rsgpu_status_string(int status);
const char *rsgpu_last_error(void);

/* ---- memory helpers ------------------------------------------------------- */
/* AllocAligned (unsafe.go:19-43): n shards of `each` bytes in one device
 * allocation, each starting on a 64-byte boundary; out[0] owns the block. */
int rsgpu_alloc_shards(rsgpu_ctx *ctx, int n, size_t each, uint8_t **out);
int rsgpu_free(rsgpu_ctx *ctx, void *device_ptr);
int rsgpu_host_alloc(size_t bytes, void **out); /* pinned host memory */
int rsgpu_host_free(void *p);
/* Synchronous copy between any host / device addresses (unified addressing). */
int rsgpu_memcpy(void *dst, const void *src, size_t bytes);

/* ---- encoder (Encoder / Extensions interfaces, reedsolomon.go:25-165) ----- */
void rsgpu_options_init(rsgpu_options *opts);
/* New (reedsolomon.go:425-601).  ctx may be NULL for a host-only encoder that
 * can plan (rsgpu_decode_plan) but not run device work. */
int rsgpu_encoder_new(rsgpu_ctx *ctx, int data_shards, int parity_shards, const rsgpu_options *opts,
                      rsgpu_encoder **out);
int rsgpu_encoder_free(rsgpu_encoder *enc);
/* DataShards / ParityShards / TotalShards / ShardSizeMultiple (reedsolomon.go:141-165) */
int rsgpu_encoder_info(const rsgpu_encoder *enc, int *data_shards, int *parity_shards,
                       int *shard_size_multiple, int *codec);
/* Leopard encoders: how many erasure patterns have their error locators
 * cached on the device (at most 256; the reference caches GF(2^8) ones,
 * leopard8.go:465-513).  0 for classic encoders. */
int rsgpu_leopard_errloc_cached(const rsgpu_encoder *enc);
/* The (k+p) x k encoding matrix of a classic encoder (reedSolomon.m). */
int rsgpu_encoder_matrix(const rsgpu_encoder *enc, uint8_t *out);

/* Encode (reedsolomon.go:686-702; leopard.go:139; leopard8.go:128) */
int rsgpu_encode(rsgpu_encoder *enc, uint8_t *const *shards, size_t shard_size);
/* EncodeIdx (reedsolomon.go:708-757): parity[o] ^= M[k+o][idx] * data */
int rsgpu_encode_idx(rsgpu_encoder *enc, const uint8_t *data_shard, int idx, uint8_t *const *parity,
                     size_t shard_size);
/* Update (reedsolomon.go:762-853): for every data shard c with new_data[c]
 * != NULL, shards[c] ^= new_data[c] (like the reference, the old shard is left
 * holding the delta) and parity ^= P[:, c] * delta.  Leopard: ErrNotSupported
 * (leopard.go:316). */
int rsgpu_update(rsgpu_encoder *enc, uint8_t *const *shards, const uint8_t *const *new_data,
                 size_t shard_size);
/* DecodeIdx (reedsolomon.go:1464-1617): progressive decoding.  expect[k+p]
 * marks the shards that will arrive as input; input[i] (NULL when not in this
 * call) contributes to every non-NULL dst[j] through the decode matrix of the
 * first k expected shards, accumulated (dst must start zeroed).  expect ==
 * NULL: merging mode, dst[i] ^= input[i].  Leopard: ErrNotSupported. */
int rsgpu_decode_idx(rsgpu_encoder *enc, uint8_t *const *dst, const uint8_t *expect,
                     const uint8_t *const *input, size_t shard_size);
/* Split (reedsolomon.go:1803-1856; leopard.go:320-370) of `len` bytes of
 * device data into k+p shards of *per_shard = ceil(len/k) bytes (Leopard:
 * rounded up to 64).  data[len, cap) may be used as spare room, like a Go
 * slice's capacity, and is zeroed.  rsgpu_split_plan gives per_shard and the
 * bytes of padding the split needs; rsgpu_split fills shards[k+p] with views
 * of `data` for the shards that fit and, for the rest, zeroed 64-byte aligned
 * slices of the caller's `padding` buffer (64-byte aligned, padding_bytes
 * long), into which the data past the last full shard is copied. */
int rsgpu_split_plan(rsgpu_encoder *enc, size_t len, size_t cap, size_t *per_shard, size_t *padding_bytes);
int rsgpu_split(rsgpu_encoder *enc, uint8_t *data, size_t len, size_t cap, uint8_t *padding,
                size_t padding_bytes, uint8_t **shards, size_t *per_shard);
/* Join (reedsolomon.go:1858-1898): copies the first out_size bytes of the
 * data shards (device, shard_size bytes each) to dst (device or host). */
int rsgpu_join(rsgpu_encoder *enc, void *dst, uint8_t *const *shards, size_t shard_size, size_t out_size);
/* Verify (reedsolomon.go:857-871; leopard.go:393-419) */
int rsgpu_verify(rsgpu_encoder *enc, uint8_t *const *shards, size_t shard_size, int *ok);
/* Reconstruct / ReconstructData / ReconstructSome (reedsolomon.go:1446,1634,1655;
 * leopard.go:378-391).  required has n_required entries (k or k+p).
 * written (optional, k+p entries) reports which shards were filled. */
int rsgpu_reconstruct(rsgpu_encoder *enc, uint8_t **shards, const uint8_t *present,
                      size_t shard_size, uint8_t *written);
int rsgpu_reconstruct_data(rsgpu_encoder *enc, uint8_t **shards, const uint8_t *present,
                           size_t shard_size, uint8_t *written);
int rsgpu_reconstruct_some(rsgpu_encoder *enc, uint8_t **shards, const uint8_t *present,
                           const uint8_t *required, int n_required, size_t shard_size,
                           uint8_t *written);

/* Asynchronous variants: enqueue on the context stream and return without
 * waiting (the caller orders later work on that stream or synchronises).
 * Missing reconstruct outputs must be preallocated (no NULL entries). */
int rsgpu_encode_async(rsgpu_encoder *enc, uint8_t *const *shards, size_t shard_size);
int rsgpu_reconstruct_async(rsgpu_encoder *enc, uint8_t *const *shards, const uint8_t *present,
                            size_t shard_size, int data_only);

/* Host-buffer variants: shards are HOST pointers; H2D/D2H happen inside,
 * pipelined in column chunks over two copy directions and the compute stream. */
int rsgpu_encode_host(rsgpu_encoder *enc, uint8_t *const *host_shards, size_t shard_size);
int rsgpu_reconstruct_host(rsgpu_encoder *enc, uint8_t **host_shards, const uint8_t *present,
                           size_t shard_size, int data_only, uint8_t *written);
/* ReconstructSome (reedsolomon.go:1655; leopard.go:386-391) on host buffers. */
int rsgpu_reconstruct_some_host(rsgpu_encoder *enc, uint8_t **host_shards, const uint8_t *present,
                                const uint8_t *required, int n_required, size_t shard_size, uint8_t *written);
/* Verify (reedsolomon.go:857-871; leopard.go:393-419) on host buffers: every
 * shard goes H2D, only the outcome comes back. */
int rsgpu_verify_host(rsgpu_encoder *enc, uint8_t *const *host_shards, size_t shard_size, int *ok);
/* EncodeIdx (reedsolomon.go:708-757) on host buffers: parity[o] ^= M[k+o][idx] * data. */
int rsgpu_encode_idx_host(rsgpu_encoder *enc, const uint8_t *host_data, int idx, uint8_t *const *host_parity,
                          size_t shard_size);
/* Update (reedsolomon.go:762-853) on host buffers, with rsgpu_update's semantics. */
int rsgpu_update_host(rsgpu_encoder *enc, uint8_t *const *host_shards, const uint8_t *const *host_new_data,
                      size_t shard_size);
/* DecodeIdx (reedsolomon.go:1464-1617) on host buffers, with rsgpu_decode_idx's semantics. */
int rsgpu_decode_idx_host(rsgpu_encoder *enc, uint8_t *const *host_dst, const uint8_t *expect,
                          const uint8_t *const *host_input, size_t shard_size);

/* Decode planning without device work: the rows codeSomeShards receives in
 * reconstruct (reedsolomon.go:1710-1779).  rows_out[n_out x k], out_idx[n_out],
 * in_idx[k] = the first k present shards.  n_out == 0: nothing to do. */
int rsgpu_decode_plan(rsgpu_encoder *enc, const uint8_t *present, int data_only,
                      const uint8_t *required, int n_required, uint8_t *rows_out, int *out_idx,
                      int *n_out, int *in_idx);

/* ---- kernel seam (galois_gen_switch_amd64.go:29-44 fn pointers) ---------- */
/* codeSomeShards (reedsolomon.go:882-975): out[o][start:stop] (^)= sum_i
 * rows[o*n_in+i] * in[i][start:stop]; clear=1 overwrites, 0 accumulates. */
int rsgpu_code_some_shards(rsgpu_ctx *ctx, const uint8_t *rows, int n_in, int n_out,
                           const uint8_t *const *in, uint8_t *const *out, size_t start, size_t stop,
                           int clear);
/* checkSomeShards (reedsolomon.go:1373-1387) fused: *ok = all(rows*in == to_check) */
int rsgpu_check_some_shards(rsgpu_ctx *ctx, const uint8_t *rows, int n_in, int n_out,
                            const uint8_t *const *in, const uint8_t *const *to_check,
                            size_t nbytes, int *ok);
/* No counterpart in the reference.  checkSomeShards for callers that cannot
 * allocate device memory (a process that reserved its whole HBM budget up
 * front, or a latency-critical path that must not risk cudaMalloc): no
 * context, no allocation.  Its scratch is one 8 MiB array per device, static in
 * the library and held until exit; more than 32 inputs need
 * n_out * round_up(nbytes, 256) <= 8 MiB - 256, larger calls return
 * RS_ERR_INVALID_INPUT.  It runs one fixed set of table kernels (never the
 * run-time compiled ones).  Runs on `cuda_stream` on the current device and
 * waits for it.  The first call on a device does the set-up that does take
 * memory: it looks up the array's device address and loads the array and
 * every kernel the calls use (CUDA loads code lazily, on first use, and
 * loading allocates); later calls on that device allocate nothing.  Make
 * that first call at start-up, before any stream capture.  Calls that
 * overlap on the GPU share the array and race: serialise them. */
int rsgpu_check_some_shards_noalloc(const uint8_t *rows, int n_in, int n_out,
                                    const uint8_t *const *in, const uint8_t *const *to_check,
                                    size_t nbytes, void *cuda_stream, int *ok);
/* galMulSlice / galMulSliceXor (galois_amd64.go:49-159; mulslice.go:29-38) */
int rsgpu_gal_mul_slice(rsgpu_ctx *ctx, uint8_t c, const uint8_t *in, uint8_t *out, size_t n,
                        int xor_into);
/* sliceXor (galois_amd64.go:162-203): out ^= in */
int rsgpu_slice_xor(rsgpu_ctx *ctx, const uint8_t *in, uint8_t *out, size_t n);

/* ---- batched execution (no counterpart in the reference, which runs one
 * Encode / Reconstruct / Verify call per stripe: reedsolomon.go:686,1670,857) */
#define RS_JOB_ENCODE 0
#define RS_JOB_RECONSTRUCT 1
#define RS_JOB_RECONSTRUCT_DATA 2
#define RS_JOB_VERIFY 3

#define RS_BATCH_PERSISTENT 0 /* one launch over every job's tiles */
#define RS_BATCH_PER_STRIPE 1 /* one launch per stripe operation (baseline) */
#define RS_BATCH_GRAPH 2      /* the per-stripe launches captured once in a CUDA graph */

typedef struct rsgpu_stripe {
    int op;                   /* RS_JOB_* */
    int data_shards, parity_shards;
    size_t shard_size;
    uint8_t *const *shards;   /* k+p device pointers; reconstruct outputs preallocated */
    const uint8_t *present;   /* reconstruct: k+p flags, 0 = missing */
} rsgpu_stripe;

typedef struct rsgpu_batch rsgpu_batch;
/* A batch of classic-codec stripe operations (k <= 32 per stripe), each
 * stripe with its own geometry, size and erasure set. */
int rsgpu_batch_create(rsgpu_ctx *ctx, const rsgpu_options *opts, rsgpu_batch **out);
int rsgpu_batch_destroy(rsgpu_batch *batch);
int rsgpu_batch_clear(rsgpu_batch *batch);
/* Plans stripes on the host (matrices, decode rows via the inversion tree). */
int rsgpu_batch_add(rsgpu_batch *batch, const rsgpu_stripe *stripes, int n);
/* Runs all planned jobs on the context stream (RS_BATCH_*); _run waits. */
int rsgpu_batch_run(rsgpu_batch *batch, int mode);
int rsgpu_batch_run_async(rsgpu_batch *batch, int mode);
/* Verify outcome per added stripe in add order (1 = parity matches). */
int rsgpu_batch_results(rsgpu_batch *batch, int *ok, int n);
/* Stripes, jobs, tiles and algorithmic bytes (reads + writes) of the batch. */
int rsgpu_batch_info(rsgpu_batch *batch, int *n_stripes, int *n_jobs, long long *n_tiles, double *bytes);
/* Tile size of the persistent launch in bytes (multiple of 4096; 0 = default). */
int rsgpu_batch_set_tile(rsgpu_batch *batch, int tile_bytes);
/* Autotuner of the persistent launch (no counterpart in the reference): runs
 * the batch's own jobs (reps timed runs per shape; every run rewrites the
 * same outputs) for tile sizes 4-64 KiB and 2-4 persistent CTAs per SM, keeps
 * the fastest shape for later runs and reports it (any out pointer may be
 * NULL). */
int rsgpu_batch_autotune(rsgpu_batch *batch, int reps, int *tile_bytes, int *ctas_per_sm, float *ms);

/* ---- StreamEncoder (streaming.go:23-700) -----------------------------------
 * Block-wise Encode / Verify / Reconstruct over caller callbacks (the
 * reference's io.Reader / io.Writer), classic codec only like rsStream.  A
 * read callback fills up to `max` bytes of shard `shard` and returns the
 * count (fewer only at the end of the stream, 0 at its end, < 0 on error); a
 * write callback returns 0 on success.  Callbacks run on the calling thread
 * while the device works on the previous block.  `block` is the per-shard
 * block size (the reference's WithStreamBlockSize, default 4 MiB).  Read and
 * write failures return RS_ERR_STREAM_READ / RS_ERR_STREAM_WRITE with the
 * shard index in *err_shard. */
typedef long long (*rsgpu_read_fn)(void *user, int shard, uint8_t *buf, size_t max);
typedef int (*rsgpu_write_fn)(void *user, int shard, const uint8_t *buf, size_t n);
/* Encode (streaming.go:209-245): reads shards 0..k-1, writes k..k+p-1. */
int rsgpu_stream_encode(rsgpu_encoder *enc, rsgpu_read_fn rd, rsgpu_write_fn wr, void *user, size_t block,
                        int *err_shard);
/* Verify (streaming.go:419-444): reads all k+p shards; *ok = 1 when every block verifies. */
int rsgpu_stream_verify(rsgpu_encoder *enc, rsgpu_read_fn rd, void *user, size_t block, int *ok, int *err_shard);
/* Reconstruct (streaming.go:453-500): reads shards with valid[i], writes the
 * rebuilt shards with fill[i]; valid and fill must not both be set. */
int rsgpu_stream_reconstruct(rsgpu_encoder *enc, const uint8_t *valid, const uint8_t *fill, rsgpu_read_fn rd,
                             rsgpu_write_fn wr, void *user, size_t block, int *err_shard);

/* ---- request server (no counterpart in the reference) --------------------
 * Continuous batching over device-resident stripes: any host thread submits
 * requests; a server thread admits them in arrival order while the bytes of
 * work in flight stay under `inflight_budget` and reconstruct outputs without
 * a caller buffer fit in an HBM arena of `arena_bytes`, and launches each
 * admitted group as one micro-batch on a free stream, so requests arriving
 * while others run are admitted as soon as a stream frees up and their work
 * overlaps on the device.  Classic and Leopard requests queue in separate
 * lanes of `streams` streams each (classic on high-priority streams); the
 * Leopard lane holds at most 3/4 of the budget, so classic requests are
 * never queued behind Leopard ones. */
typedef struct rsgpu_request {
    int op;                     /* RS_JOB_* (verify: classic stripes only) */
    int data_shards, parity_shards;
    int leopard;                /* RS_LEOPARD_* as in rsgpu_options */
    size_t shard_size;
    uint8_t **shards;           /* k+p device pointers; NULL reconstruct outputs are
                                   allocated from the arena and written back here */
    const uint8_t *present;     /* reconstruct: 0 = missing (NULL = all present) */
    uint64_t tag;               /* returned in the completion */
    int result;                 /* verify: set to 1 when parity matches */
} rsgpu_request;

typedef struct rsgpu_completion {
    uint64_t ticket, tag;
    int status;                 /* RS_OK or the request's error */
    double latency_us;          /* submit -> device completion */
    double queue_us;            /* submit -> launch (admission wait); latency_us - queue_us is service time */
} rsgpu_completion;

typedef struct rsgpu_server_stats {
    uint64_t submitted, completed, failed;
    double bytes;               /* algorithmic bytes of completed requests */
    double elapsed_s;           /* first submit -> last completion */
    double p50_us, p99_us, mean_us, max_us;
    double max_inflight_bytes;
} rsgpu_server_stats;

typedef struct rsgpu_server rsgpu_server;
int rsgpu_server_create(rsgpu_ctx *ctx, size_t arena_bytes, size_t inflight_budget, int max_batch,
                        int streams, rsgpu_server **out);
/* The request (and its shards array) must stay valid until completion. */
int rsgpu_server_submit(rsgpu_server *srv, rsgpu_request *req, uint64_t *ticket);
/* Up to `max` completions, non-blocking; returns how many. */
int rsgpu_server_poll(rsgpu_server *srv, rsgpu_completion *out, int max);
/* Frees a completed request's arena outputs and bookkeeping. */
int rsgpu_server_release(rsgpu_server *srv, uint64_t ticket);
/* Waits until nothing is queued or running; RS_ERR_TIMEOUT after timeout_ms. */
int rsgpu_server_wait_idle(rsgpu_server *srv, int timeout_ms);
int rsgpu_server_get_stats(rsgpu_server *srv, rsgpu_server_stats *out);
int rsgpu_server_reset_stats(rsgpu_server *srv);
/* Open-loop load generator: submits reqs[i] at arrival_us[i] microseconds
 * after the call from a dedicated thread; returns when all are submitted. */
int rsgpu_server_replay(rsgpu_server *srv, rsgpu_request *reqs, const double *arrival_us, int n,
                        uint64_t *tickets);
/* Drains queued and running work, then frees the server. */
int rsgpu_server_destroy(rsgpu_server *srv);

/* ---- autotuner (no counterpart in the reference: CPU dispatch there is by
 * cpuid, galois_gen_switch_amd64.go:29-44) -------------------------------- */
/* Times every GF(2^8) kernel variant on scratch buffers of the given geometry
 * (n_in <= 32, n_out <= 16) and records the fastest for that geometry and
 * size bucket; ms_out (optional) receives the per-variant milliseconds. */
int rsgpu_autotune_gf8(rsgpu_ctx *ctx, int n_in, int n_out, size_t nbytes, int mode, int reps,
                       float *ms_out, int *best_out);
/* Force one variant for every launch (-1 restores the tuned choice). */
int rsgpu_force_variant(int variant);
/* Records a tuning result without timing (e.g. one saved from an earlier
 * rsgpu_autotune_gf8): launches of this geometry, mode and size bucket use
 * `variant`; -1 removes the record (the untuned default applies again). */
int rsgpu_record_variant(int n_in, int n_out, size_t nbytes, int mode, int variant);
int rsgpu_num_variants(void);

/* ---- run-time generated XOR-network kernels (variant 7).  No counterpart
 * in the reference, whose per-shape kernels are generated at build time
 * (_gen/gen.go) and whose GFNI path applies the same 8x8 bit matrices
 * (genGFNIMatrix, galois.go:1004-1016) one coefficient at a time. -------- */
/* 1 when NVRTC is loadable and variant 7 can run, else 0. */
int rsgpu_xornet_available(void);
/* Waits for queued background compiles; returns how many XOR-network
 * kernels are compiled in this process. */
int rsgpu_xornet_sync(void);
/* Drops queued background compiles and waits (at most 30 s) for the ones
 * running; later launches of those matrices use the table kernels.  Call
 * before exiting a process that may still be compiling: NVRTC registers
 * exit handlers during its first compile, and they can run while that
 * compile is still in progress.  The Python package calls it at exit. */
int rsgpu_xornet_drain(void);
/* Compiles now the XOR-network kernels a classic encoder's Encode and Verify
 * launch (every input / output tile), so their first calls run the network
 * rather than a table kernel.  Needs no device.  Returns the number of
 * kernels ready (0 for Leopard encoders or without NVRTC). */
int rsgpu_encoder_prepare_kernels(rsgpu_encoder *enc);
/* Generated source for an n_out x n_in coefficient tile (row-major,
 * n_in <= 32, n_out <= 16) in one mode (0 write, 1 xor into the outputs,
 * 2 compare with them), factoring `group` inputs at a time (0: the default
 * for n_out): the CUDA kernel (host == 0) or the same schedule as a plain C
 * function rs_xornet_host(in, out, nchunk, flag) over host arrays
 * (host == 1).  Copies at most cap bytes including the NUL and returns the
 * full length without it, or a negative status. */
long long rsgpu_xornet_source(const uint8_t *coef, int n_in, int n_out, int mode, int group, int host,
                              char *buf, size_t cap);

/* ---- host algebra (CPU only, no device needed) --------------------------- */
/* buildMatrix* (reedsolomon.go:232-413): (total x k) row-major */
int rsgpu_build_matrix(int matrix_kind, int data_shards, int total_shards, uint8_t *out);
/* matrix.Invert (matrix.go:192-207) */
int rsgpu_invert_matrix(const uint8_t *m, int n, uint8_t *out);
/* galMultiply (galois.go:852) */
uint8_t rsgpu_gal_mul(uint8_t a, uint8_t b);

#ifdef __cplusplus
}
#endif
#endif /* RSGPU_H */
