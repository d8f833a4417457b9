// batch.cu -- batched mixed-geometry execution of many stripe operations.
//
// The reference runs one Encode / Reconstruct / Verify call per stripe
// (reedsolomon.go:686, :1670, :857); a GPU launch per stripe leaves most SMs
// idle for small stripes and pays launch latency per call.  Here every
// stripe operation becomes one GF(2^8) contraction job (<= 32 inputs, <= 8
// outputs per job; more outputs become several jobs), the jobs' byte ranges
// are cut into equal tiles, and ONE persistent launch processes all tiles.
// Consecutive tiles are grouped into units of equal cost (the larger of
// their shared-memory lookups and their HBM bytes), which the CTAs take
// from a global counter at run time: a CTA's consecutive tiles mostly share
// a job and its shared-memory product tables, and CTAs that draw slower
// tiles take fewer units, so the SMs finish together.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <map>

#include "batch_plan.h"
#include "gf8_device.cuh"
#include "rsgpu_internal.h"
#include "trace.h"

namespace rsgpu {
namespace {

using namespace gf8dev;

constexpr int kBatchOut = 8;  // outputs per job (two packed groups)

struct BatchJob {
    const uint8_t *in[kMaxIn];
    uint8_t *out[kBatchOut];
    uint8_t coef[kBatchOut][kMaxIn];
    long long nbytes;      // multiple of 16
    long long tile_begin;  // first global tile of this job
    int n_in, n_out, mode, flag;
};

struct MulArgs {
    uint32_t m[8];
};

// Inputs are read in groups of kGrp 16-byte vectors, the next group's loads
// issued before the current group's products (software pipelining: a
// thread's HBM loads otherwise wait one latency per group, and with tiles
// of a few KiB a thread has only one or two vectors per tile to overlap
// them with).  Four inputs per group up to four outputs, two with 5-8
// outputs, whose 32 accumulators leave fewer registers.
template <int G>
__device__ void batch_tile(const BatchJob &j, uint32_t tab_s, const Mul &mu, long long v0, long long v1,
                           uint32_t &mism) {
    constexpr int kGrp = G == 1 ? 4 : 2;
    const int n_in = j.n_in;
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
        uint32_t acc[G][16];
#pragma unroll
        for (int g = 0; g < G; g++)
#pragma unroll
            for (int b = 0; b < 16; b++) acc[g][b] = 0;
        uint4 cur[kGrp], nxt[kGrp];
#pragma unroll
        for (int u = 0; u < kGrp; u++) {
            cur[u] = u < n_in ? ld_in(j.in[u], v) : make_uint4(0, 0, 0, 0);
            nxt[u] = make_uint4(0, 0, 0, 0);
        }
        for (int i = 0; i < n_in; i += kGrp) {
#pragma unroll
            for (int u = 0; u < kGrp; u++)
                if (i + kGrp + u < n_in) nxt[u] = ld_in(j.in[i + kGrp + u], v);
#pragma unroll
            for (int u = 0; u < kGrp; u++)
                if (i + u < n_in) mac_vec<G, kVariantPrmt>(cur[u], tab_s + (i + u) * kInStride, mu, acc);
#pragma unroll
            for (int u = 0; u < kGrp; u++) cur[u] = nxt[u];
        }
#pragma unroll
        for (int g = 0; g < G; g++) {
            uint4 w[4];
            transpose4x4(acc[g][0], acc[g][1], acc[g][2], acc[g][3], w[0].x, w[1].x, w[2].x, w[3].x);
            transpose4x4(acc[g][4], acc[g][5], acc[g][6], acc[g][7], w[0].y, w[1].y, w[2].y, w[3].y);
            transpose4x4(acc[g][8], acc[g][9], acc[g][10], acc[g][11], w[0].z, w[1].z, w[2].z, w[3].z);
            transpose4x4(acc[g][12], acc[g][13], acc[g][14], acc[g][15], w[0].w, w[1].w, w[2].w, w[3].w);
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int oo = 4 * g + o;
                if (oo >= j.n_out) break;
                uint4 *dst = reinterpret_cast<uint4 *>(j.out[oo]) + v;
                if (j.mode == kModeWrite) {
                    __stcs(dst, w[o]);
                } else if (j.mode == kModeXor) {
                    uint4 old = __ldcs(dst);
                    old.x ^= w[o].x; old.y ^= w[o].y; old.z ^= w[o].z; old.w ^= w[o].w;
                    __stcs(dst, old);
                } else {
                    const uint4 chk = __ldcs(dst);
                    mism |= (chk.x ^ w[o].x) | (chk.y ^ w[o].y) | (chk.z ^ w[o].z) | (chk.w ^ w[o].w);
                }
            }
        }
    }
}

// Work is handed out dynamically: the tile list is cut into cost-balanced
// units of consecutive tiles (kUnitsPerCta per CTA on average), and each CTA
// takes the next unit from a global counter until none is left, so CTAs
// that drew slower tiles take fewer units.  unit_first[u] is unit u's first
// tile, unit_job[u] the job holding it; a CTA's units come in increasing
// order, and it rebuilds its tables only when a unit starts another job.
__global__ void __launch_bounds__(kThreads, 4) gf8_batch_kernel(const BatchJob *__restrict__ jobs, int njobs,
                                                             const long long *__restrict__ unit_first,
                                                             const int *__restrict__ unit_job, int n_units,
                                                             int *counter, int tile_vecs, int *flags, MulArgs mul) {
    extern __shared__ __align__(128) uint32_t smem_raw[];
    __shared__ BatchJob sj;
    __shared__ int s_job, s_unit;
    __shared__ long long s_next;
    uint32_t *tab = aligned_tables(smem_raw);
    const uint32_t tab_s = (uint32_t)__cvta_generic_to_shared(tab);
    Mul mu;
#pragma unroll
    for (int j = 0; j < 8; j++) mu.m[j] = mul.m[j];
    int job = -1;
    long long next_begin = 0;
    uint32_t mism = 0;
    for (;;) {
        __syncthreads();  // every thread has read s_unit (and s_job) of the previous unit
        if (threadIdx.x == 0) s_unit = atomicAdd(counter, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= n_units) break;
        const long long t0 = unit_first[u], t1 = unit_first[u + 1];
        for (long long t = t0; t < t1; t++) {
            if (job < 0 || t >= next_begin || t < sj.tile_begin) {
                __syncthreads();  // previous job's tables are no longer read
                if (threadIdx.x == 0) {
                    int j = job;
                    if (t == t0) j = unit_job[u];  // first tile of a unit
                    while (j + 1 < njobs && jobs[j + 1].tile_begin <= t) j++;
                    s_job = j;
                    s_next = (j + 1 < njobs) ? jobs[j + 1].tile_begin : LLONG_MAX;
                }
                __syncthreads();
                const int nj = s_job;
                next_begin = s_next;
                if (nj != job) {
                    if (mism && job >= 0 && sj.flag >= 0) flags[sj.flag] = 1;
                    mism = 0;
                    job = nj;
                    __syncthreads();
                    const uint32_t *src = reinterpret_cast<const uint32_t *>(jobs + job);
                    uint32_t *dst = reinterpret_cast<uint32_t *>(&sj);
                    for (int w = threadIdx.x; w < (int)(sizeof(BatchJob) / 4); w += blockDim.x) dst[w] = src[w];
                    __syncthreads();
                    if (sj.n_out <= 4) build_tables_from<1>(tab, sj.coef, sj.n_in, sj.n_out);
                    else build_tables_from<2>(tab, sj.coef, sj.n_in, sj.n_out);
                    __syncthreads();
                }
            }
            const long long nvec = sj.nbytes >> 4;
            const long long v0 = (t - sj.tile_begin) * tile_vecs;
            const long long v1 = v0 + tile_vecs < nvec ? v0 + tile_vecs : nvec;
            if (sj.n_out <= 4) batch_tile<1>(sj, tab_s, mu, v0, v1, mism);
            else batch_tile<2>(sj, tab_s, mu, v0, v1, mism);
        }
    }
    if (mism && job >= 0 && sj.flag >= 0) flags[sj.flag] = 1;
}

const uint32_t kMulInit[8] = {4u, 1u << 26, 1u << 18, 1u << 10, 1u << 30, 1u << 22, 1u << 14, 1u << 6};

}  // namespace
}  // namespace rsgpu

using namespace rsgpu;

struct rsgpu_batch {
    rsgpu_ctx *ctx = nullptr;
    rsgpu_options opts{};
    std::map<std::pair<int, int>, rsgpu_encoder *> encoders;
    std::vector<BatchJob> jobs;          // regular jobs (vector path)
    std::vector<BatchJob> irregular;     // misaligned / ragged jobs: per-job launches
    int n_stripes = 0;
    int tile_bytes = 0;                  // 0: default
    int ctas_per_sm = 0;                 // persistent CTAs per SM; 0: default
    bool dirty = true;
    // device state
    BatchJob *d_jobs = nullptr;
    size_t d_jobs_cap = 0;
    long long *d_cta = nullptr;  // first tile of every work unit
    size_t d_cta_cap = 0;
    int *d_ujob = nullptr;  // job of every unit's first tile
    size_t d_ujob_cap = 0;
    int n_units = 0;
    int *d_flags = nullptr;
    size_t d_flags_cap = 0;
    int grid = 0;
    long long n_tiles = 0;
    double bytes = 0;
    cudaGraphExec_t graph = nullptr;
    ~rsgpu_batch() {
        for (auto &kv : encoders) rsgpu_encoder_free(kv.second);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(d_jobs);
        cudaFree(d_cta);
        cudaFree(d_ujob);
        cudaFree(d_flags);
    }
};

namespace {

constexpr int kDefaultTile = 16384;
constexpr int kBatchBlocksPerSm = 4;
constexpr int kUnitsPerCta = 16;  // work units per persistent CTA, on average

int get_encoder(rsgpu_batch *b, int k, int p, rsgpu_encoder **out) {
    auto key = std::make_pair(k, p);
    auto it = b->encoders.find(key);
    if (it != b->encoders.end()) {
        *out = it->second;
        return RS_OK;
    }
    rsgpu_options o = b->opts;
    o.leopard = RS_LEOPARD_AS_NEEDED;
    rsgpu_encoder *e = nullptr;
    int rc = rsgpu_encoder_new(b->ctx, k, p, &o, &e);
    if (rc) return rc;
    if (e->codec != RS_CODEC_CLASSIC) {
        rsgpu_encoder_free(e);
        return RS_ERR_NOT_SUPPORTED;
    }
    b->encoders[key] = e;
    *out = e;
    return RS_OK;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// Appends jobs out[o] (^)= rows[o] . in for a stripe, 8 outputs per job.
int add_jobs(rsgpu_batch *b, const uint8_t *rows, int n_in, int n_out, const std::vector<const uint8_t *> &in,
             const std::vector<uint8_t *> &out, size_t nbytes, int mode, int flag) {
    if (n_in > kMaxIn) return RS_ERR_NOT_SUPPORTED;
    for (int o0 = 0; o0 < n_out; o0 += kBatchOut) {
        BatchJob j;
        memset(&j, 0, sizeof j);
        const int no = std::min(kBatchOut, n_out - o0);
        bool regular = (nbytes % 16) == 0;
        for (int i = 0; i < n_in; i++) {
            j.in[i] = in[i];
            regular &= aligned16(in[i]);
        }
        for (int o = 0; o < no; o++) {
            j.out[o] = out[o0 + o];
            regular &= aligned16(out[o0 + o]);
            for (int i = 0; i < n_in; i++) j.coef[o][i] = rows[(size_t)(o0 + o) * n_in + i];
        }
        j.nbytes = (long long)nbytes;
        j.n_in = n_in;
        j.n_out = no;
        j.mode = mode;
        j.flag = flag;
        (regular ? b->jobs : b->irregular).push_back(j);
    }
    return RS_OK;
}

// Cost-balanced units of consecutive tiles (cost: see job_cost; the cut:
// batch_plan.h), about kUnitsPerCta per CTA, handed out at run time
// (gf8_batch_kernel); unit_first has n_units + 1 entries, unit_job the job
// of each unit's first tile.
void plan_tiles(rsgpu_batch *b, std::vector<long long> &unit_first, std::vector<int> &unit_job) {
    const int tile = b->tile_bytes > 0 ? b->tile_bytes : kDefaultTile;
    long long t = 0;
    std::vector<double> job_cost(b->jobs.size());
    b->bytes = 0;
    for (size_t i = 0; i < b->jobs.size(); i++) {
        BatchJob &j = b->jobs[i];
        j.tile_begin = t;
        const long long nt = (j.nbytes + tile - 1) / tile;
        t += nt;
        const int rw = j.n_in + j.n_out * (j.mode == kModeWrite ? 1 : 2);
        // Time per byte column: the larger of the shared-memory lookups
        // (two per input byte and output group of four, 32 per clock per SM)
        // and the HBM bytes (about 22 per clock per SM at the measured copy
        // rate), in units of one group's lookups per input byte.
        const int groups = (j.n_out + 3) / 4;
        job_cost[i] = std::max((double)j.n_in * groups, 0.72 * rw) * (double)j.nbytes;
        b->bytes += (double)rw * (double)j.nbytes;
    }
    b->n_tiles = t;
    // resident CTAs per SM of the batch kernel, queried once per device
    static std::atomic<int> resident_by_dev[64];
    const int dev = b->ctx->info.device & 63;
    int resident = resident_by_dev[dev].load(std::memory_order_relaxed);
    if (resident == 0) {
        const size_t smem = (size_t)kMaxIn * kInStride + kTableAlign;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, (const void *)gf8_batch_kernel, kThreads,
                                                          smem) != cudaSuccess || resident < 1)
            resident = 1;
        resident_by_dev[dev].store(resident, std::memory_order_relaxed);
    }
    const int per_sm = std::min(resident, b->ctas_per_sm > 0 ? b->ctas_per_sm : kBatchBlocksPerSm);
    const int grid = std::max(1, (int)std::min<long long>(t, (long long)b->ctx->info.sm_count * per_sm));
    b->grid = grid;
    const int n_units = (int)std::max(1LL, std::min<long long>(t, (long long)grid * kUnitsPerCta));
    b->n_units = n_units;
    std::vector<long long> begins(b->jobs.size()), counts(b->jobs.size());
    for (size_t i = 0; i < b->jobs.size(); i++) {
        begins[i] = b->jobs[i].tile_begin;
        counts[i] = (b->jobs[i].nbytes + tile - 1) / tile;
    }
    BatchUnitPlan plan = plan_batch_units(begins, counts, job_cost, n_units);
    unit_first = std::move(plan.unit_first);
    unit_job = std::move(plan.unit_job);
}

// Uploads the job table and CTA ranges, stream-ordered on `st`: growing a
// device buffer uses cudaFreeAsync and the context's stream-ordered pool
// (doubling), never a device-wide synchronising cudaFree, so a request
// server can plan one slot's micro-batch while other streams keep running.
int upload(rsgpu_batch *b, cudaStream_t st) {
    if (!b->dirty) return RS_OK;
    std::vector<long long> unit_first;
    std::vector<int> unit_job;
    plan_tiles(b, unit_first, unit_job);
    cudaMemPool_t pool = b->ctx->pool;
    auto grow = [st, pool](auto *&ptr, size_t &cap, size_t want) -> cudaError_t {
        if (want <= cap) return cudaSuccess;
        want = std::max(want, 2 * cap);
        if (ptr) {
            cudaError_t e = cudaFreeAsync(ptr, st);
            if (e != cudaSuccess) return e;
        }
        ptr = nullptr;
        cap = 0;
        cudaError_t e = cudaMallocFromPoolAsync((void **)&ptr, want, pool, st);
        if (e == cudaSuccess) cap = want;
        return e;
    };
    RS_CUDA(grow(b->d_jobs, b->d_jobs_cap, std::max<size_t>(1, b->jobs.size()) * sizeof(BatchJob)));
    RS_CUDA(grow(b->d_cta, b->d_cta_cap, unit_first.size() * sizeof(long long)));
    RS_CUDA(grow(b->d_ujob, b->d_ujob_cap, unit_job.size() * sizeof(int)));
    // the stripes' flags, then the unit counter of the persistent launch
    RS_CUDA(grow(b->d_flags, b->d_flags_cap, (std::max(1, b->n_stripes) + 1) * sizeof(int)));
    if (!b->jobs.empty())
        RS_CUDA(cudaMemcpyAsync(b->d_jobs, b->jobs.data(), b->jobs.size() * sizeof(BatchJob), cudaMemcpyHostToDevice,
                                st));
    RS_CUDA(cudaMemcpyAsync(b->d_cta, unit_first.data(), unit_first.size() * sizeof(long long),
                            cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(b->d_ujob, unit_job.data(), unit_job.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->dirty = false;
    return RS_OK;
}

int launch_persistent(rsgpu_batch *b, cudaStream_t st) {
    if (b->jobs.empty()) return RS_OK;
    const int tile = b->tile_bytes > 0 ? b->tile_bytes : kDefaultTile;
    const size_t smem = (size_t)kMaxIn * kInStride + kTableAlign;
    MulArgs mul;
    for (int i = 0; i < 8; i++) mul.m[i] = kMulInit[i];
    int *counter = b->d_flags + std::max(1, b->n_stripes);  // zeroed with the flags before every run
    gf8_batch_kernel<<<b->grid, kThreads, smem, st>>>(b->d_jobs, (int)b->jobs.size(), b->d_cta, b->d_ujob,
                                                     b->n_units, counter, tile / 16, b->d_flags, mul);
    RS_CUDA(cudaGetLastError());
    return RS_OK;
}

// One launch per job through the per-call path (the baseline).
int launch_per_job(rsgpu_batch *b, cudaStream_t st, const std::vector<BatchJob> &list) {
    for (const BatchJob &j : list) {
        GfMatArgs a;
        std::vector<const uint8_t *> in(j.in, j.in + j.n_in);
        std::vector<uint8_t *> out(j.out, j.out + j.n_out);
        fill_args(a, &j.coef[0][0], kMaxIn, j.n_in, j.n_out, in.data(), out.data(), (size_t)j.nbytes,
                  j.flag >= 0 ? b->d_flags + j.flag : b->d_flags);
        RS_CUDA(launch_gf8_tile(st, b->ctx->info, a, j.mode, choose_variant(j.n_in, j.n_out, j.mode, (size_t)j.nbytes)));
    }
    return RS_OK;
}

}  // namespace

extern "C" {

int rsgpu_batch_create(rsgpu_ctx *ctx, const rsgpu_options *opts, rsgpu_batch **out) {
    if (!ctx || !out) return RS_ERR_INVALID_INPUT;
    auto *b = new rsgpu_batch();
    b->ctx = ctx;
    if (opts) b->opts = *opts;
    else rsgpu_options_init(&b->opts);
    *out = b;
    return RS_OK;
}

int rsgpu_batch_destroy(rsgpu_batch *b) {
    delete b;
    return RS_OK;
}

int rsgpu_batch_clear(rsgpu_batch *b) {
    if (!b) return RS_ERR_INVALID_INPUT;
    b->jobs.clear();
    b->irregular.clear();
    b->n_stripes = 0;
    b->dirty = true;
    return RS_OK;
}

int rsgpu_batch_set_tile(rsgpu_batch *b, int tile_bytes) {
    if (!b || tile_bytes < 0 || (tile_bytes % 4096) != 0) return RS_ERR_INVALID_INPUT;
    b->tile_bytes = tile_bytes;
    b->dirty = true;
    return RS_OK;
}

int rsgpu_batch_autotune(rsgpu_batch *b, int reps, int *tile_out, int *ctas_out, float *ms_out) {
    RS_TRACE("rsgpu_batch_autotune");
    if (!b) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::recursive_mutex> lk(b->ctx->mu);
    if (b->jobs.empty()) return RS_ERR_SHARD_NO_DATA;
    if (reps < 1) reps = 2;
    cudaStream_t st = b->ctx->stream;
    cudaEvent_t e0, e1;
    RS_CUDA(cudaEventCreate(&e0));
    RS_CUDA(cudaEventCreate(&e1));
    static const int kTiles[] = {4096, 8192, 16384, 32768, 65536};
    static const int kCtas[] = {2, 3, 4};
    float best = 1e30f;
    int best_tile = kDefaultTile, best_ctas = kBatchBlocksPerSm, rc = RS_OK;
    for (int ctas : kCtas)
        for (int tile : kTiles) {
            b->tile_bytes = tile;
            b->ctas_per_sm = ctas;
            b->dirty = true;
            rc = batch_run_on(b, RS_BATCH_PERSISTENT, st);  // plans, uploads and warms this shape
            if (rc) break;
            float ms = 0;
            if (cudaEventRecord(e0, st) != cudaSuccess) { rc = RS_ERR_CUDA; break; }
            for (int r = 0; r < reps && !rc; r++) rc = batch_run_on(b, RS_BATCH_PERSISTENT, st);
            if (rc) break;
            if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = RS_ERR_CUDA;
                break;
            }
            ms /= reps;
            if (ms < best) {
                best = ms;
                best_tile = tile;
                best_ctas = ctas;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tile_bytes = best_tile;
    b->ctas_per_sm = best_ctas;
    b->dirty = true;
    if (rc) return rc;
    if (tile_out) *tile_out = best_tile;
    if (ctas_out) *ctas_out = best_ctas;
    if (ms_out) *ms_out = best;
    return RS_OK;
}

int rsgpu_batch_add(rsgpu_batch *b, const rsgpu_stripe *s, int n) {
    if (!b || (!s && n > 0)) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::recursive_mutex> lk(b->ctx->mu);
    for (int idx = 0; idx < n; idx++) {
        const rsgpu_stripe &st = s[idx];
        rsgpu_encoder *e = nullptr;
        int rc = get_encoder(b, st.data_shards, st.parity_shards, &e);
        if (rc) return rc;
        if (st.shard_size == 0) return RS_ERR_SHARD_NO_DATA;
        if (!st.shards) return RS_ERR_TOO_FEW_SHARDS;
        const int k = e->k, p = e->p;
        const int flag = b->n_stripes;
        if (st.op == RS_JOB_ENCODE || st.op == RS_JOB_VERIFY) {
            std::vector<const uint8_t *> in(st.shards, st.shards + k);
            std::vector<uint8_t *> out(st.shards + k, st.shards + k + p);
            for (auto *q : in) if (!q) return RS_ERR_SHARD_SIZE;
            for (auto *q : out) if (!q) return RS_ERR_SHARD_SIZE;
            rc = add_jobs(b, e->parity_rows.data(), k, p, in, out, st.shard_size,
                          st.op == RS_JOB_ENCODE ? kModeWrite : kModeVerify, flag);
        } else if (st.op == RS_JOB_RECONSTRUCT || st.op == RS_JOB_RECONSTRUCT_DATA) {
            if (!st.present) return RS_ERR_INVALID_INPUT;
            std::vector<uint8_t> rows;
            std::vector<int> out_idx, in_idx;
            rc = classic_decode_plan(e, st.present, st.op == RS_JOB_RECONSTRUCT_DATA, nullptr, 0, rows, out_idx,
                                     in_idx);
            if (rc) return rc;
            if (!out_idx.empty()) {
                std::vector<const uint8_t *> in;
                std::vector<uint8_t *> out;
                for (int i : in_idx) {
                    if (!st.shards[i]) return RS_ERR_SHARD_SIZE;
                    in.push_back(st.shards[i]);
                }
                for (int o : out_idx) {
                    if (!st.shards[o]) return RS_ERR_INVALID_INPUT;  // outputs are preallocated
                    out.push_back(st.shards[o]);
                }
                rc = add_jobs(b, rows.data(), k, (int)out.size(), in, out, st.shard_size, kModeWrite, flag);
            }
        } else {
            return RS_ERR_INVALID_INPUT;
        }
        if (rc) return rc;
        b->n_stripes++;
    }
    b->dirty = true;
    return RS_OK;
}

int rsgpu_batch_run_async(rsgpu_batch *b, int mode) {
    RS_TRACE("rsgpu_batch_run_async");
    if (!b) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::recursive_mutex> lk(b->ctx->mu);
    return batch_run_on(b, mode, b->ctx->stream);
}

}  // extern "C"

int rsgpu::batch_stripe_count(const rsgpu_batch *b) { return b->n_stripes; }

int rsgpu::batch_read_flags(rsgpu_batch *b, int *ok, int n, cudaStream_t st) {
    if (n <= 0) return RS_OK;
    std::vector<int> flags(n);
    RS_CUDA(cudaMemcpyAsync(flags.data(), b->d_flags, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; i++) ok[i] = flags[i] == 0;
    return RS_OK;
}

int rsgpu::batch_run_on(rsgpu_batch *b, int mode, cudaStream_t st) {
    rsgpu_ctx *ctx = b->ctx;
    int rc = upload(b, st);
    if (rc) return rc;
    // the stripes' flags and the persistent launch's unit counter
    RS_CUDA(cudaMemsetAsync(b->d_flags, 0, (std::max(1, b->n_stripes) + 1) * sizeof(int), st));
    if (mode == RS_BATCH_PERSISTENT) {
        rc = launch_persistent(b, st);
        if (rc) return rc;
        return launch_per_job(b, st, b->irregular);
    }
    if (mode == RS_BATCH_PER_STRIPE) {
        rc = launch_per_job(b, st, b->jobs);
        if (rc) return rc;
        return launch_per_job(b, st, b->irregular);
    }
    if (mode == RS_BATCH_GRAPH) {
        if (!b->graph) {
            // capture on the context's own stream, replay on the current one
            cudaStream_t cs = ctx->own_stream;
            RS_CUDA(cudaStreamSynchronize(st));
            RS_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
            int r1 = launch_per_job(b, cs, b->jobs);
            int r2 = r1 ? r1 : launch_per_job(b, cs, b->irregular);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(cs, &g);
            if (r2) {
                if (g) cudaGraphDestroy(g);
                return r2;
            }
            RS_CUDA(e);
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            RS_CUDA(e);
        }
        RS_CUDA(cudaGraphLaunch(b->graph, st));
        return RS_OK;
    }
    return RS_ERR_INVALID_INPUT;
}

extern "C" {

int rsgpu_batch_run(rsgpu_batch *b, int mode) {
    int rc = rsgpu_batch_run_async(b, mode);
    if (rc) return rc;
    RS_CUDA(cudaStreamSynchronize(b->ctx->stream));
    return RS_OK;
}

int rsgpu_batch_results(rsgpu_batch *b, int *ok, int n) {
    if (!b || !ok || n < 0 || n > b->n_stripes) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::recursive_mutex> lk(b->ctx->mu);
    if (n == 0) return RS_OK;
    std::vector<int> flags(n);
    RS_CUDA(cudaStreamSynchronize(b->ctx->stream));
    RS_CUDA(cudaMemcpy(flags.data(), b->d_flags, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) ok[i] = flags[i] == 0;
    return RS_OK;
}

int rsgpu_batch_info(rsgpu_batch *b, int *n_stripes, int *n_jobs, long long *n_tiles, double *bytes) {
    if (!b) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::recursive_mutex> lk(b->ctx->mu);
    int rc = upload(b, b->ctx->stream);
    if (rc) return rc;
    if (n_stripes) *n_stripes = b->n_stripes;
    if (n_jobs) *n_jobs = (int)(b->jobs.size() + b->irregular.size());
    if (n_tiles) *n_tiles = b->n_tiles;
    if (bytes) {
        double irr = 0;
        for (const BatchJob &j : b->irregular)
            irr += (double)(j.n_in + j.n_out * (j.mode == kModeWrite ? 1 : 2)) * (double)j.nbytes;
        *bytes = b->bytes + irr;
    }
    return RS_OK;
}

}  // extern "C"
