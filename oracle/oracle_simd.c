/*
 * oracle_simd.c -- the reference's x86 SIMD kernel algorithms, restated for
 * the timed CPU baseline.  TEST / BENCH INFRASTRUCTURE ONLY (never shipped).
 *
 * Algorithms restated (from the generator sources, not the generated asm):
 *   GFNI:  genGFNIMatrix (galois.go:950-964) turns each coefficient into an
 *          8x8 GF(2) affine matrix; the mulGFNI_IxO_64 kernels
 *          (_gen/gen.go:858-1083) load each 64-byte input vector once and
 *          accumulate VGF2P8AFFINEQB products into O register accumulators.
 *   AVX2:  genCodeGenMatrix (galois.go:914-946) builds 16-entry low/high
 *          nibble product tables; mulAvxTwo_IxO (_gen/gen.go:339-598) splits
 *          each 32-byte vector into nibbles and combines two VPSHUFB lookups.
 *   Threads split the byte range into 64-byte aligned pieces like
 *   codeSomeShardsP (reedsolomon.go:979-1068).
 * Results are checked against the scalar oracle in tests/test_oracle_kats.py.
 */
#include "oracle.h"

#include <immintrin.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static int simd_level = -1; /* 0 scalar, 1 avx2, 2 avx512+gfni */

int ora_simd_level(void) {
    if (simd_level < 0) {
        __builtin_cpu_init();
        if (__builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx512f") &&
            __builtin_cpu_supports("avx512bw"))
            simd_level = 2;
        else if (__builtin_cpu_supports("avx2"))
            simd_level = 1;
        else
            simd_level = 0;
    }
    return simd_level;
}

typedef struct {
    const uint8_t *rows;
    int n_in, n_out;
    const uint8_t *const *in;
    uint8_t *const *out;
    size_t start, stop;
    int clear;
    int level;
    const uint64_t *gfni;   /* [n_in][n_out] */
    const uint8_t *nib;     /* [n_in][n_out][32]: 16 low | 16 high */
} job_t;

#define OUT_GROUP 16

__attribute__((target("avx512f,avx512bw,gfni")))
static void run_gfni(const job_t *j) {
    size_t off = j->start;
    for (; off + 64 <= j->stop; off += 64) {
        for (int o0 = 0; o0 < j->n_out; o0 += OUT_GROUP) {
            int no = j->n_out - o0 < OUT_GROUP ? j->n_out - o0 : OUT_GROUP;
            __m512i acc[OUT_GROUP];
            for (int o = 0; o < no; o++)
                acc[o] = j->clear ? _mm512_setzero_si512() : _mm512_loadu_si512(j->out[o0 + o] + off);
            for (int i = 0; i < j->n_in; i++) {
                __m512i v = _mm512_loadu_si512(j->in[i] + off);
                const uint64_t *mrow = j->gfni + (size_t)i * j->n_out + o0;
                for (int o = 0; o < no; o++)
                    acc[o] = _mm512_xor_si512(
                        acc[o], _mm512_gf2p8affine_epi64_epi8(v, _mm512_set1_epi64((long long)mrow[o]), 0));
            }
            for (int o = 0; o < no; o++) _mm512_storeu_si512(j->out[o0 + o] + off, acc[o]);
        }
    }
    if (off < j->stop) {
        for (int o = 0; o < j->n_out; o++)
            for (int i = 0; i < j->n_in; i++)
                ora_gal_mul_slice(j->rows[o * j->n_in + i], j->in[i] + off, j->out[o] + off,
                                  j->stop - off, !(i == 0 && j->clear));
    }
}

__attribute__((target("avx2")))
static void run_avx2(const job_t *j) {
    const __m256i mask = _mm256_set1_epi8(0x0f);
    size_t off = j->start;
    for (; off + 32 <= j->stop; off += 32) {
        for (int o0 = 0; o0 < j->n_out; o0 += OUT_GROUP) {
            int no = j->n_out - o0 < OUT_GROUP ? j->n_out - o0 : OUT_GROUP;
            __m256i acc[OUT_GROUP];
            for (int o = 0; o < no; o++)
                acc[o] = j->clear ? _mm256_setzero_si256()
                                  : _mm256_loadu_si256((const __m256i *)(j->out[o0 + o] + off));
            for (int i = 0; i < j->n_in; i++) {
                __m256i v = _mm256_loadu_si256((const __m256i *)(j->in[i] + off));
                __m256i lo = _mm256_and_si256(v, mask);
                __m256i hi = _mm256_and_si256(_mm256_srli_epi64(v, 4), mask);
                for (int o = 0; o < no; o++) {
                    const uint8_t *t = j->nib + ((size_t)i * j->n_out + o0 + o) * 32;
                    __m256i tl = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)t));
                    __m256i th = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)(t + 16)));
                    acc[o] = _mm256_xor_si256(acc[o], _mm256_xor_si256(_mm256_shuffle_epi8(tl, lo),
                                                                       _mm256_shuffle_epi8(th, hi)));
                }
            }
            for (int o = 0; o < no; o++) _mm256_storeu_si256((__m256i *)(j->out[o0 + o] + off), acc[o]);
        }
    }
    if (off < j->stop) {
        for (int o = 0; o < j->n_out; o++)
            for (int i = 0; i < j->n_in; i++)
                ora_gal_mul_slice(j->rows[o * j->n_in + i], j->in[i] + off, j->out[o] + off,
                                  j->stop - off, !(i == 0 && j->clear));
    }
}

static void run_scalar(const job_t *j) {
    for (int o = 0; o < j->n_out; o++)
        for (int i = 0; i < j->n_in; i++)
            ora_gal_mul_slice(j->rows[o * j->n_in + i], j->in[i] + j->start, j->out[o] + j->start,
                              j->stop - j->start, !(i == 0 && j->clear));
}

static void *worker(void *arg) {
    const job_t *j = (const job_t *)arg;
    /* process in L2-sized rounds like perRound (reedsolomon.go:493-537) */
    const size_t round = 32 * 1024;
    job_t sub = *j;
    for (size_t s = j->start; s < j->stop; s += round) {
        sub.start = s;
        sub.stop = s + round < j->stop ? s + round : j->stop;
        if (j->level == 2) run_gfni(&sub);
        else if (j->level == 1) run_avx2(&sub);
        else run_scalar(&sub);
    }
    return NULL;
}

int ora_code_some_shards_fast(const uint8_t *rows, int n_in, int n_out, const uint8_t *const *in,
                              uint8_t *const *out, size_t nbytes, int clear, int threads) {
    if (n_out == 0 || nbytes == 0) return ORA_OK;
    if (threads < 1) threads = 1;
    int level = ora_simd_level();
    uint64_t *gfni = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n_in * n_out);
    uint8_t *nib = (uint8_t *)malloc((size_t)n_in * n_out * 32);
    for (int i = 0; i < n_in; i++)
        for (int o = 0; o < n_out; o++) {
            uint8_t c = rows[o * n_in + i];
            gfni[(size_t)i * n_out + o] = ora_gfni_matrix(c);
            for (int x = 0; x < 16; x++) {
                nib[((size_t)i * n_out + o) * 32 + x] = ora_gal_mul(c, (uint8_t)x);
                nib[((size_t)i * n_out + o) * 32 + 16 + x] = ora_gal_mul(c, (uint8_t)(x << 4));
            }
        }
    size_t per = (nbytes + (size_t)threads - 1) / (size_t)threads;
    per = (per + 63) & ~(size_t)63;
    pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    job_t *jobs = (job_t *)malloc(sizeof(job_t) * (size_t)threads);
    int started = 0;
    for (int t = 0; t < threads; t++) {
        size_t s = (size_t)t * per;
        if (s >= nbytes) break;
        jobs[t] = (job_t){rows, n_in, n_out, in, out, s, s + per < nbytes ? s + per : nbytes,
                          clear, level, gfni, nib};
        if (threads == 1) worker(&jobs[t]);
        else pthread_create(&tid[t], NULL, worker, &jobs[t]);
        started++;
    }
    if (threads > 1)
        for (int t = 0; t < started; t++) pthread_join(tid[t], NULL);
    free(tid);
    free(jobs);
    free(gfni);
    free(nib);
    return ORA_OK;
}
