/*
 * oracle.h -- CPU restatement of klauspost/reedsolomon's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the
 * smoke() entry point and bench.py's cpu_baseline / reference arm load it.
 * The product library (reedsolomon_b200/librsgpu.so) never links it.
 *
 * Parity of this restatement is pinned against the reference's own golden
 * vectors (galois.go literal tables, galois_test.go / matrix_test.go /
 * reedsolomon_test.go / leopard*_test.go known answers and the
 * gf2p811dMulMatrices* fixtures); see tests/test_oracle_kats.py.
 * Leopard encode/decode bytes have no reference KAT: they are pinned through
 * the field tables (leopard8.go:1271 GFNI matrices) plus round trips.
 *
 * Return codes follow the product's rs_status values (include/rsgpu.h).
 */
#ifndef RS_ORACLE_H
#define RS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORA_OK = 0,
    ORA_ERR_TOO_FEW_SHARDS = -1,
    ORA_ERR_SHARD_NO_DATA = -2,
    ORA_ERR_SHARD_SIZE = -3,
    ORA_ERR_INVALID_SHARD_SIZE = -4,
    ORA_ERR_INV_SHARD_NUM = -5,
    ORA_ERR_MAX_SHARD_NUM = -6,
    ORA_ERR_NOT_SUPPORTED = -7,
    ORA_ERR_INVALID_INPUT = -8,
    ORA_ERR_RECONSTRUCT_REQUIRED = -9,
    ORA_ERR_SINGULAR = -10,
    ORA_ERR_NOT_SQUARE = -11,
    ORA_ERR_SHORT_DATA = -12,
};

/* matrix kinds (options.go:252-303 WithJerasureMatrix / WithPAR1Matrix / WithCauchyMatrix / WithFastOneParityMatrix) */
enum { ORA_MAT_DEFAULT = 0, ORA_MAT_CAUCHY = 1, ORA_MAT_PAR1 = 2, ORA_MAT_JERASURE = 3, ORA_MAT_XOR = 4 };

/* ---- GF(2^8), poly 0x11D (galois.go) ---- */
void ora_gf8_tables(uint8_t log_out[256], uint8_t exp_out[256], uint8_t inv_out[256],
                    uint8_t low_out[256 * 16], uint8_t high_out[256 * 16]);
void ora_gf8_multable(uint8_t out[65536]);
uint8_t ora_gal_mul(uint8_t a, uint8_t b);
uint8_t ora_gal_exp(uint8_t a, int n);
uint8_t ora_gal_divide(uint8_t a, uint8_t b);
uint64_t ora_gfni_matrix(uint8_t c);

/* ---- matrix algebra (matrix.go) ---- */
int ora_mat_invert(const uint8_t *m, int n, uint8_t *out);
void ora_mat_multiply(const uint8_t *a, int ar, int ac, const uint8_t *b, int bc, uint8_t *out);
int ora_build_matrix(int kind, int data_shards, int total_shards, uint8_t *out);

/* ---- kernels (galois_noasm.go semantics) ---- */
void ora_gal_mul_slice(uint8_t c, const uint8_t *in, uint8_t *out, size_t n, int xor_into);
void ora_code_some_shards(const uint8_t *rows, int n_in, int n_out, const uint8_t *const *in,
                          uint8_t *const *out, size_t nbytes, int clear);

/* ---- classic codec (reedsolomon.go) ---- */
int ora_rs_encode(int k, int p, int kind, uint8_t *const *shards, size_t size);
int ora_rs_encode_idx(int k, int p, int kind, const uint8_t *data, int idx, uint8_t *const *parity,
                      size_t size);
int ora_rs_verify(int k, int p, int kind, uint8_t *const *shards, size_t size, int *ok);
/* present[i]!=0 marks shard i as holding data; missing outputs must be preallocated
 * (size bytes).  required may be NULL; n_required = its length (k or k+p). */
int ora_rs_reconstruct(int k, int p, int kind, uint8_t *const *shards, const uint8_t *present,
                       size_t size, int data_only, const uint8_t *required, int n_required,
                       uint8_t *written);
int ora_split(int k, int p, int leopard, const uint8_t *data, size_t len, size_t *per_shard, uint8_t *out);
int ora_join(int k, const uint8_t *const *shards, const size_t *sizes, int n_shards, uint8_t *dst,
             size_t out_size);
int ora_rs_update(int k, int p, int kind, uint8_t *const *shards, const uint8_t *const *new_data,
                  size_t size);
int ora_rs_decode_idx(int k, int p, int kind, uint8_t *const *dst, const uint8_t *expect,
                      const uint8_t *const *input, size_t size);
int ora_rs_decode_rows(int k, int p, int kind, const uint8_t *present, int data_only,
                       const uint8_t *required, int n_required, uint8_t *rows_out,
                       int *out_idx, int *n_out, int *in_idx);

/* ---- Leopard GF(2^16) (leopard.go) ---- */
void ora_leo16_tables(uint16_t *log_out, uint16_t *exp_out, uint16_t *skew_out,
                      uint16_t *walsh_out);
uint16_t ora_leo16_mullog(uint16_t a, uint16_t log_b);
/* CPU-baseline timing only: 1 switches the Leopard products to AVX2
 * nibble-table multiplies (when the CPU has AVX2), 0 back to the scalar
 * restatement; returns whether the AVX2 path is on. */
int ora_leo_simd(int on);
int ora_leo16_encode(int k, int p, uint8_t *const *shards, size_t size);
int ora_leo16_reconstruct(int k, int p, uint8_t *const *shards, const uint8_t *present,
                          size_t size, int recover_all, uint8_t *written);
int ora_leo16_errlocs(int k, int p, const uint8_t *present, uint16_t *errlocs_out);
int ora_leo16_verify(int k, int p, uint8_t *const *shards, size_t size, int *ok);

/* ---- Leopard GF(2^8) (leopard8.go) ---- */
void ora_leo8_tables(uint8_t *log_out, uint8_t *exp_out, uint8_t *skew_out, uint8_t *walsh_out);
uint8_t ora_leo8_mullog(uint8_t a, uint8_t log_b);
uint64_t ora_leo8_gfni_matrix(uint8_t log_m);
int ora_leo8_encode(int k, int p, uint8_t *const *shards, size_t size);
int ora_leo8_reconstruct(int k, int p, uint8_t *const *shards, const uint8_t *present,
                         size_t size, int recover_all, uint8_t *written);
int ora_leo8_errlocs(int k, int p, const uint8_t *present, uint8_t *errlocs_out);
int ora_leo8_verify(int k, int p, uint8_t *const *shards, size_t size, int *ok);

/* ---- CPU baseline: the reference's SIMD algorithms restated (see oracle_simd.c) ---- */
int ora_simd_level(void);
int ora_code_some_shards_fast(const uint8_t *rows, int n_in, int n_out, const uint8_t *const *in,
                              uint8_t *const *out, size_t nbytes, int clear, int threads);

#ifdef __cplusplus
}
#endif
#endif
