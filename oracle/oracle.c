/*
 * oracle.c -- CPU restatement of klauspost/reedsolomon's hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker that tests/, smoke() and the
 * CPU-baseline legs of bench.py compare the CUDA product against.  It is never
 * linked into the product library.  Every function cites the reference file
 * and lines whose behaviour it restates; chunking and SIMD dispatch in the
 * reference are results-neutral (all ops are column-local) and are omitted.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* GF(2^8) with generating polynomial 29 (x^8+x^4+x^3+x^2+1)                  */
/* galois.go:14-27 (constants), :29 logTable, :71 expTable, :78 invTable,     */
/* :80 mulTable, :337/:593 mulTableLow/High; gentables.go:59-131 generators.  */
/* ------------------------------------------------------------------------ */
static uint8_t g_log[256], g_exp[256], g_inv[256];
static uint8_t g_mul[256][256];
static int g_gf8_ready;

static void gf8_init(void) {
    if (g_gf8_ready) return;
    unsigned x = 1;
    for (int i = 0; i < 255; i++) {
        g_exp[i] = (uint8_t)x;
        x <<= 1;
        if (x & 0x100) x ^= 0x100 | 29;
    }
    g_exp[255] = g_exp[0]; /* galois.go:66 "Entry 255 is the same as entry 0" */
    g_log[0] = 0;          /* galois.go:30 literal */
    for (int i = 0; i < 255; i++) g_log[g_exp[i]] = (uint8_t)i;
    for (int a = 0; a < 256; a++)
        for (int b = 0; b < 256; b++)
            g_mul[a][b] = (a == 0 || b == 0) ? 0 : g_exp[(g_log[a] + g_log[b]) % 255];
    g_inv[0] = 0;
    for (int a = 1; a < 256; a++) g_inv[a] = g_exp[(255 - g_log[a]) % 255];
    g_gf8_ready = 1;
}

void ora_gf8_tables(uint8_t log_out[256], uint8_t exp_out[256], uint8_t inv_out[256],
                    uint8_t low_out[256 * 16], uint8_t high_out[256 * 16]) {
    gf8_init();
    memcpy(log_out, g_log, 256);
    memcpy(exp_out, g_exp, 256);
    memcpy(inv_out, g_inv, 256);
    /* gentables.go:107-131 generateMulTableHalf */
    for (int a = 0; a < 256; a++)
        for (int b = 0; b < 16; b++) {
            low_out[a * 16 + b] = g_mul[a][b];
            high_out[a * 16 + b] = g_mul[a][b << 4];
        }
}

void ora_gf8_multable(uint8_t out[65536]) {
    gf8_init();
    memcpy(out, g_mul, 65536);
}

uint8_t ora_gal_mul(uint8_t a, uint8_t b) { gf8_init(); return g_mul[a][b]; }

/* galois.go:898-912 galExp */
uint8_t ora_gal_exp(uint8_t a, int n) {
    gf8_init();
    if (n == 0) return 1;
    if (a == 0) return 0;
    int lr = (int)g_log[a] * n;
    while (lr >= 255) lr -= 255;
    return g_exp[(uint8_t)lr];
}

/* galois.go:870-885 galDivide */
uint8_t ora_gal_divide(uint8_t a, uint8_t b) {
    gf8_init();
    if (a == 0 || b == 0) return 0;
    int lr = (int)g_log[a] - (int)g_log[b];
    if (lr < 0) lr += 255;
    return g_exp[(uint8_t)lr];
}

/* galois.go:887-894 galOneOver */
static uint8_t gal_one_over(uint8_t a) { return g_exp[(uint8_t)(g_log[a] ^ 255)]; }

/* The 8x8 GF(2) affine matrix of "multiply by c" in the bit layout of
 * galois.go:948 gf2p811dMulMatrices (byte 7-j of the word drives output bit j). */
uint64_t ora_gfni_matrix(uint8_t c) {
    gf8_init();
    uint64_t m = 0;
    for (int ib = 0; ib < 8; ib++) {
        uint8_t r = g_mul[c][1 << ib];
        for (int ob = 0; ob < 8; ob++)
            if ((r >> ob) & 1) m |= (uint64_t)1 << ((7 - ob) * 8 + ib);
    }
    return m;
}

/* ------------------------------------------------------------------------ */
/* Matrix algebra, row-major uint8 arrays (matrix.go)                         */
/* ------------------------------------------------------------------------ */

/* matrix.go:103-117 Multiply: out[ar x bc] = a[ar x ac] * b[ac x bc] */
void ora_mat_multiply(const uint8_t *a, int ar, int ac, const uint8_t *b, int bc, uint8_t *out) {
    gf8_init();
    for (int r = 0; r < ar; r++)
        for (int c = 0; c < bc; c++) {
            uint8_t v = 0;
            for (int i = 0; i < ac; i++) v ^= g_mul[a[r * ac + i]][b[i * bc + c]];
            out[r * bc + c] = v;
        }
}

/* matrix.go:192-265 Invert + gaussianElimination on [m | I] */
int ora_mat_invert(const uint8_t *m, int n, uint8_t *out) {
    gf8_init();
    int cols = 2 * n;
    uint8_t *w = (uint8_t *)calloc((size_t)n * cols, 1);
    uint8_t *tmp = (uint8_t *)malloc((size_t)cols);
    for (int r = 0; r < n; r++) {
        memcpy(w + r * cols, m + r * n, (size_t)n);
        w[r * cols + n + r] = 1;
    }
    for (int r = 0; r < n; r++) {
        if (w[r * cols + r] == 0) {
            for (int below = r + 1; below < n; below++) {
                if (w[below * cols + r] != 0) {
                    memcpy(tmp, w + r * cols, cols);
                    memcpy(w + r * cols, w + below * cols, cols);
                    memcpy(w + below * cols, tmp, cols);
                    break;
                }
            }
        }
        if (w[r * cols + r] == 0) {
            free(w);
            free(tmp);
            return ORA_ERR_SINGULAR;
        }
        if (w[r * cols + r] != 1) {
            uint8_t s = gal_one_over(w[r * cols + r]);
            for (int c = 0; c < cols; c++) w[r * cols + c] = g_mul[w[r * cols + c]][s];
        }
        for (int below = r + 1; below < n; below++) {
            uint8_t s = w[below * cols + r];
            if (s != 0)
                for (int c = 0; c < cols; c++) w[below * cols + c] ^= g_mul[s][w[r * cols + c]];
        }
    }
    for (int d = 0; d < n; d++)
        for (int above = 0; above < d; above++) {
            uint8_t s = w[above * cols + d];
            if (s != 0)
                for (int c = 0; c < cols; c++) w[above * cols + c] ^= g_mul[s][w[d * cols + c]];
        }
    for (int r = 0; r < n; r++) memcpy(out + r * n, w + r * cols + n, (size_t)n);
    free(w);
    free(tmp);
    return ORA_OK;
}

/* matrix.go:270-281 vandermonde */
static void vandermonde(int rows, int cols, uint8_t *out) {
    for (int r = 0; r < rows; r++)
        for (int c = 0; c < cols; c++) out[r * cols + c] = ora_gal_exp((uint8_t)r, c);
}

/* reedsolomon.go:232-256 buildMatrix */
static int build_default(int k, int total, uint8_t *out) {
    uint8_t *vm = (uint8_t *)malloc((size_t)total * k);
    uint8_t *top = (uint8_t *)malloc((size_t)k * k);
    uint8_t *inv = (uint8_t *)malloc((size_t)k * k);
    vandermonde(total, k, vm);
    memcpy(top, vm, (size_t)k * k);
    int rc = ora_mat_invert(top, k, inv);
    if (rc == ORA_OK) ora_mat_multiply(vm, total, k, inv, k, out);
    free(vm);
    free(top);
    free(inv);
    return rc;
}

/* reedsolomon.go:263-337 buildMatrixJerasure */
static int build_jerasure(int k, int total, uint8_t *vm) {
    vandermonde(total, k, vm);
#define VM(r, c) vm[(r) * k + (c)]
    VM(0, 0) = 1;
    for (int i = 1; i < k; i++) VM(0, i) = 0;
    for (int i = 0; i < k - 1; i++) VM(total - 1, i) = 0;
    VM(total - 1, k - 1) = 1;
    uint8_t *tmprow = (uint8_t *)malloc((size_t)k);
    for (int i = 0; i < k; i++) {
        int r = i;
        while (r < total && VM(r, i) == 0) r++;
        if (r != i) {
            memcpy(tmprow, &VM(r, 0), k);
            memcpy(&VM(r, 0), &VM(i, 0), k);
            memcpy(&VM(i, 0), tmprow, k);
        }
        if (VM(i, i) != 1) {
            uint8_t t = gal_one_over(VM(i, i));
            for (int j = 0; j < total; j++) VM(j, i) = g_mul[VM(j, i)][t];
        }
        for (int j = 0; j < k; j++) {
            uint8_t t = VM(i, j);
            if (j != i && t != 0)
                for (int rr = 0; rr < total; rr++) VM(rr, j) ^= g_mul[t][VM(rr, i)];
        }
    }
    for (int j = 0; j < k; j++) {
        uint8_t t = VM(k, j);
        if (t != 1) {
            t = gal_one_over(t);
            for (int i = k; i < total; i++) VM(i, j) = g_mul[VM(i, j)][t];
        }
    }
    for (int i = k + 1; i < total; i++) {
        uint8_t t = VM(i, 0);
        if (t != 1) {
            t = gal_one_over(t);
            for (int j = 0; j < k; j++) VM(i, j) = g_mul[VM(i, j)][t];
        }
    }
#undef VM
    free(tmprow);
    return ORA_OK;
}

int ora_build_matrix(int kind, int k, int total, uint8_t *out) {
    gf8_init();
    if (k <= 0 || total < k) return ORA_ERR_INV_SHARD_NUM;
    memset(out, 0, (size_t)total * k);
    switch (kind) {
    case ORA_MAT_DEFAULT:
        return build_default(k, total, out);
    case ORA_MAT_JERASURE:
        return build_jerasure(k, total, out);
    case ORA_MAT_CAUCHY: /* reedsolomon.go:369-387 */
        for (int r = 0; r < total; r++)
            for (int c = 0; c < k; c++)
                out[r * k + c] = r < k ? (r == c) : g_inv[(uint8_t)(r ^ c)];
        return ORA_OK;
    case ORA_MAT_PAR1: /* reedsolomon.go:348-367 */
        for (int r = 0; r < total; r++)
            for (int c = 0; c < k; c++)
                out[r * k + c] = r < k ? (r == c) : ora_gal_exp((uint8_t)(c + 1), r - k);
        return ORA_OK;
    case ORA_MAT_XOR: /* reedsolomon.go:391-413 */
        if (total != k + 1) return ORA_ERR_INVALID_INPUT;
        for (int r = 0; r < total; r++)
            for (int c = 0; c < k; c++) out[r * k + c] = r < k ? (r == c) : 1;
        return ORA_OK;
    }
    return ORA_ERR_INVALID_INPUT;
}

/* ------------------------------------------------------------------------ */
/* Slice kernels: galois_noasm.go:9-32 galMulSlice, :45-67 galMulSliceXor,    */
/* reedsolomon.go:882-975 codeSomeShards (first input clears when clear).      */
/* ------------------------------------------------------------------------ */
void ora_gal_mul_slice(uint8_t c, const uint8_t *in, uint8_t *out, size_t n, int xor_into) {
    gf8_init();
    const uint8_t *t = g_mul[c];
    if (xor_into)
        for (size_t i = 0; i < n; i++) out[i] ^= t[in[i]];
    else
        for (size_t i = 0; i < n; i++) out[i] = t[in[i]];
}

void ora_code_some_shards(const uint8_t *rows, int n_in, int n_out, const uint8_t *const *in,
                          uint8_t *const *out, size_t nbytes, int clear) {
    gf8_init();
    for (int o = 0; o < n_out; o++)
        for (int i = 0; i < n_in; i++)
            ora_gal_mul_slice(rows[o * n_in + i], in[i], out[o], nbytes, !(i == 0 && clear));
}

/* ------------------------------------------------------------------------ */
/* Classic codec (reedsolomon.go)                                              */
/* ------------------------------------------------------------------------ */
static int classic_matrix(int k, int p, int kind, uint8_t **m_out) {
    if (k <= 0 || p < 0) return ORA_ERR_INV_SHARD_NUM;
    if (k + p > 256) return ORA_ERR_MAX_SHARD_NUM;
    uint8_t *m = (uint8_t *)malloc((size_t)(k + p) * k);
    int rc = ora_build_matrix(kind, k, k + p, m);
    if (rc != ORA_OK) {
        free(m);
        return rc;
    }
    *m_out = m;
    return ORA_OK;
}

/* reedsolomon.go:686-702 Encode */
int ora_rs_encode(int k, int p, int kind, uint8_t *const *shards, size_t size) {
    uint8_t *m;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) return rc;
    if (p > 0) ora_code_some_shards(m + (size_t)k * k, k, p, (const uint8_t *const *)shards,
                                    shards + k, size, 1);
    free(m);
    return ORA_OK;
}

/* reedsolomon.go:708-757 EncodeIdx: parity[o] ^= P[o][idx] * data */
int ora_rs_encode_idx(int k, int p, int kind, const uint8_t *data, int idx, uint8_t *const *parity,
                      size_t size) {
    uint8_t *m;
    if (p == 0) return ORA_OK;
    if (idx < 0 || idx >= k) return ORA_ERR_INV_SHARD_NUM;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) return rc;
    for (int o = 0; o < p; o++) ora_gal_mul_slice(m[(k + o) * k + idx], data, parity[o], size, 1);
    free(m);
    return ORA_OK;
}

/* reedsolomon.go:857-871 Verify + :1373-1387 checkSomeShards */
int ora_rs_verify(int k, int p, int kind, uint8_t *const *shards, size_t size, int *ok) {
    uint8_t *m;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) return rc;
    *ok = 1;
    uint8_t *tmp = (uint8_t *)malloc(size ? size : 1);
    for (int o = 0; o < p && *ok; o++) {
        uint8_t *outs[1] = {tmp};
        ora_code_some_shards(m + (size_t)(k + o) * k, k, 1, (const uint8_t *const *)shards, outs,
                             size, 1);
        if (memcmp(tmp, shards[k + o], size) != 0) *ok = 0;
    }
    free(tmp);
    free(m);
    return ORA_OK;
}

/* reedsolomon.go:620-631 multiplyRowWithMatrix */
static void row_times_matrix(const uint8_t *row, const uint8_t *mat, int k, uint8_t *out) {
    for (int j = 0; j < k; j++) {
        uint8_t v = 0;
        for (int i = 0; i < k; i++) v ^= g_mul[row[i]][mat[i * k + j]];
        out[j] = v;
    }
}

/* reedsolomon.go:1670-1781 reconstruct (decision logic + decode rows).
 * Fills rows_out[n_out x k], out_idx[n_out] (shard index written) and
 * in_idx[k] (the first k present shards, in index order).  n_out=0 with
 * ORA_OK means "nothing to do".  A required[] shorter than k+p is read as
 * false past its end (the reference indexes past it, reedsolomon.go:1690-1696). */
int ora_rs_decode_rows(int k, int p, int kind, const uint8_t *present, int data_only,
                       const uint8_t *required, int n_required, uint8_t *rows_out, int *out_idx,
                       int *n_out, int *in_idx) {
    int total = k + p;
    *n_out = 0;
    if (required && n_required < k) return ORA_ERR_TOO_FEW_SHARDS;
    int number_present = 0, data_present = 0, missing_required = 0;
    for (int i = 0; i < total; i++) {
        if (present[i]) {
            number_present++;
            if (i < k) data_present++;
        } else if (required) {
            if (i < n_required && required[i]) missing_required++;
        }
    }
    if (number_present == 0) return ORA_ERR_SHARD_NO_DATA;
    if (number_present == total || (data_only && data_present == k) ||
        (required && missing_required == 0))
        return ORA_OK;
    if (number_present < k) return ORA_ERR_TOO_FEW_SHARDS;
    uint8_t *m;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) return rc;
    int sub = 0;
    for (int r = 0; r < total && sub < k; r++)
        if (present[r]) in_idx[sub++] = r;
    uint8_t *subm = (uint8_t *)malloc((size_t)k * k);
    uint8_t *dec = (uint8_t *)malloc((size_t)k * k);
    for (int r = 0; r < k; r++) memcpy(subm + r * k, m + (size_t)in_idx[r] * k, k);
    rc = ora_mat_invert(subm, k, dec);
    if (rc == ORA_OK) {
        int cnt = 0;
        for (int i = 0; i < k; i++)
            if (!present[i] && (!required || (i < n_required && required[i]))) {
                memcpy(rows_out + (size_t)cnt * k, dec + (size_t)i * k, k);
                out_idx[cnt++] = i;
            }
        if (!data_only)
            for (int i = k; i < total; i++)
                if (!present[i] && (!required || (i < n_required && required[i]))) {
                    row_times_matrix(m + (size_t)i * k, dec, k, rows_out + (size_t)cnt * k);
                    out_idx[cnt++] = i;
                }
        *n_out = cnt;
    }
    free(subm);
    free(dec);
    free(m);
    return rc;
}

int ora_rs_reconstruct(int k, int p, int kind, uint8_t *const *shards, const uint8_t *present,
                       size_t size, int data_only, const uint8_t *required, int n_required,
                       uint8_t *written) {
    int total = k + p;
    if (k <= 0 || p < 0) return ORA_ERR_INV_SHARD_NUM;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    uint8_t *rows = (uint8_t *)malloc((size_t)total * k + 1);
    int *out_idx = (int *)malloc(sizeof(int) * (size_t)total);
    int *in_idx = (int *)malloc(sizeof(int) * (size_t)k);
    int n_out = 0;
    int rc = ora_rs_decode_rows(k, p, kind, present, data_only, required, n_required, rows, out_idx,
                                &n_out, in_idx);
    if (written) memset(written, 0, (size_t)total);
    if (rc == ORA_OK && n_out > 0) {
        const uint8_t **ins = (const uint8_t **)malloc(sizeof(void *) * (size_t)k);
        uint8_t **outs = (uint8_t **)malloc(sizeof(void *) * (size_t)n_out);
        for (int i = 0; i < k; i++) ins[i] = shards[in_idx[i]];
        for (int o = 0; o < n_out; o++) {
            outs[o] = shards[out_idx[o]];
            if (written) written[out_idx[o]] = 1;
        }
        ora_code_some_shards(rows, k, n_out, ins, outs, size, 1);
        free(ins);
        free(outs);
    }
    free(rows);
    free(out_idx);
    free(in_idx);
    return rc;
}

/* reedsolomon.go:762-853 Update / updateParityShards: for every data shard c
 * with new data, old[c] ^= new[c] (the reference overwrites the old shard
 * with the delta), then parity[o] ^= M[k+o][c] * old[c]. */
int ora_rs_update(int k, int p, int kind, uint8_t *const *shards, const uint8_t *const *new_data,
                  size_t size) {
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    int any = 0;
    for (int i = 0; i < k; i++) {
        if (new_data[i]) {
            any = 1;
            if (!shards[i]) return ORA_ERR_INVALID_INPUT;
        }
    }
    if (!any) return ORA_ERR_SHARD_NO_DATA;
    for (int o = 0; o < p; o++)
        if (!shards[k + o]) return ORA_ERR_INVALID_INPUT;
    if (p == 0) return ORA_OK;
    uint8_t *m;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) return rc;
    for (int c = 0; c < k; c++) {
        if (!new_data[c]) continue;
        for (size_t j = 0; j < size; j++) shards[c][j] ^= new_data[c][j];
        for (int o = 0; o < p; o++) ora_gal_mul_slice(m[(size_t)(k + o) * k + c], shards[c], shards[k + o], size, 1);
    }
    free(m);
    return ORA_OK;
}

/* reedsolomon.go:1464-1617 DecodeIdx.  expect == NULL: merging mode, dst[i]
 * ^= input[i].  Otherwise the decode matrix of the first k expected shards
 * (inverse of their encoding rows), one row per non-NULL dst (data rows from
 * the inverse, parity rows as parity row x inverse), restricted to the
 * columns whose input is present in this call, accumulated into dst. */
int ora_rs_decode_idx(int k, int p, int kind, uint8_t *const *dst, const uint8_t *expect,
                      const uint8_t *const *input, size_t size) {
    const int total = k + p;
    if (!expect) {
        for (int i = 0; i < total; i++)
            if (input[i] && !dst[i]) return ORA_ERR_INVALID_INPUT;
        for (int i = 0; i < total; i++)
            if (input[i])
                for (size_t j = 0; j < size; j++) dst[i][j] ^= input[i][j];
        return ORA_OK;
    }
    for (int i = 0; i < total; i++)
        if (input[i] && !expect[i]) return ORA_ERR_INVALID_INPUT;
    for (int i = 0; i < total; i++)
        if (expect[i] && dst[i]) return ORA_ERR_INVALID_INPUT;
    int *valid = (int *)malloc(sizeof(int) * (size_t)total);
    int nv = 0;
    for (int i = 0; i < total; i++)
        if (expect[i]) valid[nv++] = i;
    if (nv < k) {
        free(valid);
        return ORA_ERR_TOO_FEW_SHARDS;
    }
    uint8_t *m;
    int rc = classic_matrix(k, p, kind, &m);
    if (rc) {
        free(valid);
        return rc;
    }
    uint8_t *subm = (uint8_t *)malloc((size_t)k * k), *dec = (uint8_t *)malloc((size_t)k * k);
    for (int r = 0; r < k; r++) memcpy(subm + (size_t)r * k, m + (size_t)valid[r] * k, k);
    rc = ora_mat_invert(subm, k, dec);
    if (rc == ORA_OK) {
        uint8_t *row = (uint8_t *)malloc((size_t)k);
        for (int d = 0; d < total; d++) {
            if (!dst[d]) continue;
            if (d < k) memcpy(row, dec + (size_t)d * k, k);
            else row_times_matrix(m + (size_t)d * k, dec, k, row);
            /* columns beyond the first k valid shards carry zero coefficients */
            for (int col = 0; col < k; col++) {
                const uint8_t *in = input[valid[col]];
                if (in) ora_gal_mul_slice(row[col], in, dst[d], size, 1);
            }
        }
        free(row);
    }
    free(subm);
    free(dec);
    free(m);
    free(valid);
    return rc;
}

/* reedsolomon.go:1803-1856 Split / leopard.go:320-370 (leopard: per-shard
 * size rounded up to 64): writes the k+p shards, each per_shard bytes, one
 * after the other into out (total * per_shard bytes).  `cap` >= len models the
 * slice capacity the reference reuses (its bytes past len are zeroed); the
 * content of the shards does not depend on where each one lives. */
int ora_split(int k, int p, int leopard, const uint8_t *data, size_t len, size_t *per_shard, uint8_t *out) {
    const int total = k + p;
    if (len == 0) return ORA_ERR_SHORT_DATA;
    size_t per = (len + (size_t)k - 1) / (size_t)k;
    if (leopard) per = (per + 63) / 64 * 64;
    if (total == 1 && (!leopard || (len & 63) == 0)) per = len;
    *per_shard = per;
    if (!out) return ORA_OK;
    memset(out, 0, per * (size_t)total);
    memcpy(out, data, len);
    return ORA_OK;
}

/* reedsolomon.go:1858-1898 Join: the first out_size bytes of the data shards. */
int ora_join(int k, const uint8_t *const *shards, const size_t *sizes, int n_shards, uint8_t *dst,
             size_t out_size) {
    if (n_shards < k) return ORA_ERR_TOO_FEW_SHARDS;
    size_t have = 0;
    for (int i = 0; i < k; i++) {
        if (!shards[i]) return ORA_ERR_RECONSTRUCT_REQUIRED;
        have += sizes[i];
        if (have >= out_size) break;
    }
    if (have < out_size) return ORA_ERR_SHORT_DATA;
    size_t write = out_size, off = 0;
    for (int i = 0; i < k && write; i++) {
        const size_t n = write < sizes[i] ? write : sizes[i];
        memcpy(dst + off, shards[i], n);
        off += n;
        write -= n;
    }
    return ORA_OK;
}

/* ------------------------------------------------------------------------ */
/* Leopard GF(2^16) (leopard.go)                                               */
/* ------------------------------------------------------------------------ */
#define L16_ORDER 65536u
#define L16_MOD 65535u
static uint16_t *l16_log, *l16_exp, *l16_skew, *l16_walsh;
static uint16_t **l16_lut; /* lazily built mul16LUT per log_m: Lo[256] then Hi[256] */

/* leopard.go:1001-1006 addMod, :1009-1014 subMod (Go uint is 64-bit) */
static inline uint16_t add_mod16(uint16_t a, uint16_t b) {
    uint64_t s = (uint64_t)a + b;
    return (uint16_t)(s + (s >> 16));
}
static inline uint16_t sub_mod16(uint16_t a, uint16_t b) {
    uint64_t d = (uint64_t)a - (uint64_t)b;
    return (uint16_t)(d + (d >> 16));
}

/* leopard.go:984-998 mulLog */
static inline uint16_t mullog16(uint16_t a, uint16_t log_b) {
    if (a == 0) return 0;
    return l16_exp[add_mod16(l16_log[a], log_b)];
}

/* leopard.go:1025-1060 fwht (truncated to groups starting below mtrunc) */
static void fwht16(uint16_t *data, unsigned mtrunc) {
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= L16_ORDER) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            for (unsigned off = r; off < r + dist; off++) {
                uint16_t t0 = data[off], t1 = data[off + dist], t2 = data[off + 2 * dist],
                         t3 = data[off + 3 * dist];
                uint16_t a, b;
                a = add_mod16(t0, t1); b = sub_mod16(t0, t1); t0 = a; t1 = b;
                a = add_mod16(t2, t3); b = sub_mod16(t2, t3); t2 = a; t3 = b;
                a = add_mod16(t0, t2); b = sub_mod16(t0, t2); t0 = a; t2 = b;
                a = add_mod16(t1, t3); b = sub_mod16(t1, t3); t1 = a; t3 = b;
                data[off] = t0; data[off + dist] = t1; data[off + 2 * dist] = t2; data[off + 3 * dist] = t3;
            }
        }
        dist = dist4;
        dist4 <<= 2;
    }
}

static void leo16_init(void) {
    if (l16_log) return;
    static const uint16_t cantor[16] = {0x0001, 0xACCA, 0x3C0E, 0x163E, 0xC582, 0xED2E,
                                        0x914C, 0x4012, 0x6C98, 0x10D8, 0x6A72, 0xB900,
                                        0xFDB8, 0xFB34, 0xFF38, 0x991E}; /* leopard.go:1105-1110 */
    uint16_t *lg = (uint16_t *)calloc(L16_ORDER, 2), *ex = (uint16_t *)calloc(L16_ORDER, 2);
    /* leopard.go:1104-1147 initLUTs */
    unsigned state = 1;
    for (unsigned i = 0; i < L16_MOD; i++) {
        ex[state] = (uint16_t)i;
        state <<= 1;
        if (state >= L16_ORDER) state ^= 0x1002D;
    }
    ex[0] = L16_MOD;
    lg[0] = 0;
    for (int i = 0; i < 16; i++) {
        unsigned width = 1u << i;
        for (unsigned j = 0; j < width; j++) lg[j + width] = lg[j] ^ cantor[i];
    }
    for (unsigned i = 0; i < L16_ORDER; i++) lg[i] = ex[lg[i]];
    for (unsigned i = 0; i < L16_ORDER; i++) ex[lg[i]] = (uint16_t)i;
    ex[L16_MOD] = ex[0];
    l16_log = lg;
    l16_exp = ex;
    /* leopard.go:1150-1195 initFFTSkew */
    uint16_t temp[15];
    uint16_t *skew = (uint16_t *)calloc(L16_MOD, 2);
    uint16_t *walsh = (uint16_t *)calloc(L16_ORDER, 2);
    for (int i = 1; i < 16; i++) temp[i - 1] = (uint16_t)(1u << i);
    for (int m = 0; m < 15; m++) {
        unsigned step = 1u << (m + 1);
        skew[(1u << m) - 1] = 0;
        for (int i = m; i < 15; i++) {
            unsigned s = 1u << (i + 1);
            for (unsigned j = (1u << m) - 1; j < s; j += step) skew[j + s] = skew[j] ^ temp[i];
        }
        temp[m] = (uint16_t)(L16_MOD - lg[mullog16(temp[m], lg[temp[m] ^ 1])]);
        for (int i = m + 1; i < 15; i++) {
            uint16_t sum = add_mod16(lg[temp[i] ^ 1], temp[m]);
            temp[i] = mullog16(temp[i], sum);
        }
    }
    for (unsigned i = 0; i < L16_MOD; i++) skew[i] = lg[skew[i]];
    for (unsigned i = 0; i < L16_ORDER; i++) walsh[i] = lg[i];
    walsh[0] = 0;
    fwht16(walsh, L16_ORDER);
    l16_skew = skew;
    l16_walsh = walsh;
    l16_lut = (uint16_t **)calloc(L16_ORDER, sizeof(uint16_t *));
}

/* leopard.go:1197-1218 initMul16LUT for one log_m */
static const uint16_t *lut16(uint16_t log_m) {
    if (!l16_lut[log_m]) {
        uint16_t tmp[64];
        for (int nib = 0, shift = 0; nib < 4; nib++, shift += 4)
            for (int x = 0; x < 16; x++) tmp[nib * 16 + x] = mullog16((uint16_t)(x << shift), log_m);
        uint16_t *t = (uint16_t *)malloc(512 * 2);
        for (int i = 0; i < 256; i++) {
            t[i] = tmp[i & 15] ^ tmp[(i >> 4) + 16];
            t[256 + i] = tmp[(i & 15) + 32] ^ tmp[(i >> 4) + 48];
        }
        l16_lut[log_m] = t;
    }
    return l16_lut[log_m];
}

void ora_leo16_tables(uint16_t *log_out, uint16_t *exp_out, uint16_t *skew_out,
                      uint16_t *walsh_out) {
    leo16_init();
    if (log_out) memcpy(log_out, l16_log, L16_ORDER * 2);
    if (exp_out) memcpy(exp_out, l16_exp, L16_ORDER * 2);
    if (skew_out) memcpy(skew_out, l16_skew, L16_MOD * 2);
    if (walsh_out) memcpy(walsh_out, l16_walsh, L16_ORDER * 2);
}

uint16_t ora_leo16_mullog(uint16_t a, uint16_t log_b) {
    leo16_init();
    return mullog16(a, log_b);
}

static void xor_into_avx2(uint8_t *out, const uint8_t *in, size_t n);
static int leo_simd;

static inline void xor_into(uint8_t *out, const uint8_t *in, size_t n) {
#if defined(__x86_64__) || defined(__i386__)
    if (leo_simd) {
        xor_into_avx2(out, in, n);
        return;
    }
#endif
    for (size_t i = 0; i < n; i++) out[i] ^= in[i];
}

/* CPU-baseline only (bench.py's Leopard CPU leg): AVX2 nibble-table
 * multiplies, the approach of the reference's mulgf16 / mulgf8 AVX2 kernels
 * (_gen/gf16.go, _gen/gf8.go: each input nibble selects a 16-entry table of
 * the product's low and high output bytes with PSHUFB).  Off unless
 * ora_leo_simd(1) is called; the checker's products stay the scalar
 * refMulAdd / refMul restatements below, and a CPU test requires both to give
 * the same bytes. */
int ora_leo_simd(int on) {
#if defined(__x86_64__) || defined(__i386__)
    leo_simd = on && __builtin_cpu_supports("avx2");
#else
    leo_simd = 0;
    (void)on;
#endif
    return leo_simd;
}

#if defined(__x86_64__) || defined(__i386__)
#include <immintrin.h>
/* out ^= in (sliceXor, galois_amd64.go:162-203, with AVX2) */
__attribute__((target("avx2"))) static void xor_into_avx2(uint8_t *out, const uint8_t *in, size_t n) {
    size_t i = 0;
    for (; i + 32 <= n; i += 32)
        _mm256_storeu_si256((__m256i *)(out + i), _mm256_xor_si256(_mm256_loadu_si256((const __m256i *)(out + i)),
                                                                    _mm256_loadu_si256((const __m256i *)(in + i))));
    for (; i < n; i++) out[i] ^= in[i];
}
/* x (^)= y*log_m over whole 64-byte chunks; t: the refMulAdd table of log_m.
 * Nibble q of a symbol (bits 4q..4q+3) picks t[e], t[e << 4], t[256 + e] or
 * t[256 + (e << 4)] for q = 0..3 (refMul's table is the XOR of two nibble
 * tables per input byte). */
__attribute__((target("avx2"))) static void muladd16_avx2(uint8_t *x, const uint8_t *y, const uint16_t *t,
                                                          size_t n, int accumulate) {
    uint8_t tb[8][16];
    for (int e = 0; e < 16; e++) {
        const uint16_t v[4] = {t[e], t[e << 4], t[256 + e], t[256 + (e << 4)]};
        for (int q = 0; q < 4; q++) {
            tb[2 * q][e] = (uint8_t)v[q];
            tb[2 * q + 1][e] = (uint8_t)(v[q] >> 8);
        }
    }
    __m256i T[8];
    for (int i = 0; i < 8; i++) T[i] = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)tb[i]));
    const __m256i m4 = _mm256_set1_epi8(0x0F);
    for (size_t off = 0; off + 64 <= n; off += 64) {
        const __m256i lo = _mm256_loadu_si256((const __m256i *)(y + off));
        const __m256i hi = _mm256_loadu_si256((const __m256i *)(y + off + 32));
        const __m256i n0 = _mm256_and_si256(lo, m4), n1 = _mm256_and_si256(_mm256_srli_epi64(lo, 4), m4);
        const __m256i n2 = _mm256_and_si256(hi, m4), n3 = _mm256_and_si256(_mm256_srli_epi64(hi, 4), m4);
        __m256i plo = _mm256_xor_si256(_mm256_xor_si256(_mm256_shuffle_epi8(T[0], n0), _mm256_shuffle_epi8(T[2], n1)),
                                       _mm256_xor_si256(_mm256_shuffle_epi8(T[4], n2), _mm256_shuffle_epi8(T[6], n3)));
        __m256i phi = _mm256_xor_si256(_mm256_xor_si256(_mm256_shuffle_epi8(T[1], n0), _mm256_shuffle_epi8(T[3], n1)),
                                       _mm256_xor_si256(_mm256_shuffle_epi8(T[5], n2), _mm256_shuffle_epi8(T[7], n3)));
        if (accumulate) {
            plo = _mm256_xor_si256(plo, _mm256_loadu_si256((const __m256i *)(x + off)));
            phi = _mm256_xor_si256(phi, _mm256_loadu_si256((const __m256i *)(x + off + 32)));
        }
        _mm256_storeu_si256((__m256i *)(x + off), plo);
        _mm256_storeu_si256((__m256i *)(x + off + 32), phi);
    }
}

/* x (^)= t[y] bytewise, t: a 256-entry GF(2^8) product table (linear, so
 * t[y] = t[y & 15] ^ t[y & 0xF0]). */
__attribute__((target("avx2"))) static void muladd8_avx2(uint8_t *x, const uint8_t *y, const uint8_t *t, size_t n,
                                                         int accumulate) {
    uint8_t tl[16], th[16];
    for (int e = 0; e < 16; e++) {
        tl[e] = t[e];
        th[e] = t[e << 4];
    }
    const __m256i TL = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)tl));
    const __m256i TH = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)th));
    const __m256i m4 = _mm256_set1_epi8(0x0F);
    size_t i = 0;
    for (; i + 32 <= n; i += 32) {
        const __m256i v = _mm256_loadu_si256((const __m256i *)(y + i));
        __m256i r = _mm256_xor_si256(_mm256_shuffle_epi8(TL, _mm256_and_si256(v, m4)),
                                     _mm256_shuffle_epi8(TH, _mm256_and_si256(_mm256_srli_epi64(v, 4), m4)));
        if (accumulate) r = _mm256_xor_si256(r, _mm256_loadu_si256((const __m256i *)(x + i)));
        _mm256_storeu_si256((__m256i *)(x + i), r);
    }
    for (; i < n; i++) x[i] = (uint8_t)((accumulate ? x[i] : 0) ^ t[y[i]]);
}
#endif

/* leopard.go:907-925 refMulAdd: x ^= y*log_m on 64-byte chunks (32 lo | 32 hi) */
static void muladd16(uint8_t *x, const uint8_t *y, uint16_t log_m, size_t n) {
    const uint16_t *t = lut16(log_m);
#if defined(__x86_64__) || defined(__i386__)
    if (leo_simd) {
        muladd16_avx2(x, y, t, n, 1);
        return;
    }
#endif
    for (size_t off = 0; off + 64 <= n; off += 64)
        for (int i = 0; i < 32; i++) {
            uint16_t prod = t[y[off + i]] ^ t[256 + y[off + 32 + i]];
            x[off + i] ^= (uint8_t)prod;
            x[off + 32 + i] ^= (uint8_t)(prod >> 8);
        }
}
/* leopard.go:966-981 refMul: x = y*log_m */
static void mul16(uint8_t *x, const uint8_t *y, uint16_t log_m, size_t n) {
    const uint16_t *t = lut16(log_m);
#if defined(__x86_64__) || defined(__i386__)
    if (leo_simd) {
        muladd16_avx2(x, y, t, n, 0);
        return;
    }
#endif
    for (size_t off = 0; off + 64 <= n; off += 64)
        for (int i = 0; i < 32; i++) {
            uint16_t prod = t[y[off + i]] ^ t[256 + y[off + 32 + i]];
            x[off + i] = (uint8_t)prod;
            x[off + 32 + i] = (uint8_t)(prod >> 8);
        }
}

/* galois_noasm.go:94-98 fftDIT2 and :108-112 ifftDIT2 */
static void fft2_16(uint8_t *x, uint8_t *y, uint16_t lm, size_t n) { muladd16(x, y, lm, n); xor_into(y, x, n); }
static void ifft2_16(uint8_t *x, uint8_t *y, uint16_t lm, size_t n) { xor_into(y, x, n); muladd16(x, y, lm, n); }

/* leopard.go:739-761 fftDIT4Ref */
static void fft4_16(uint8_t **w, unsigned dist, uint16_t m01, uint16_t m23, uint16_t m02, size_t n) {
    if (m02 == L16_MOD) { xor_into(w[2 * dist], w[0], n); xor_into(w[3 * dist], w[dist], n); }
    else { fft2_16(w[0], w[2 * dist], m02, n); fft2_16(w[dist], w[3 * dist], m02, n); }
    if (m01 == L16_MOD) xor_into(w[dist], w[0], n); else fft2_16(w[0], w[dist], m01, n);
    if (m23 == L16_MOD) xor_into(w[3 * dist], w[2 * dist], n); else fft2_16(w[2 * dist], w[3 * dist], m23, n);
}
/* leopard.go:875-897 ifftDIT4Ref */
static void ifft4_16(uint8_t **w, unsigned dist, uint16_t m01, uint16_t m23, uint16_t m02, size_t n) {
    if (m01 == L16_MOD) xor_into(w[dist], w[0], n); else ifft2_16(w[0], w[dist], m01, n);
    if (m23 == L16_MOD) xor_into(w[3 * dist], w[2 * dist], n); else ifft2_16(w[2 * dist], w[3 * dist], m23, n);
    if (m02 == L16_MOD) { xor_into(w[2 * dist], w[0], n); xor_into(w[3 * dist], w[dist], n); }
    else { ifft2_16(w[0], w[2 * dist], m02, n); ifft2_16(w[dist], w[3 * dist], m02, n); }
}

/* leopard.go:764-873 ifftDITEncoder (plain copy path; the fused SIMD path is equivalent) */
static void ifft_encoder16(uint8_t *const *data, unsigned mtrunc, uint8_t **work, uint8_t **xor_res,
                           unsigned m, const uint16_t *skew, size_t n) {
    for (unsigned i = 0; i < mtrunc; i++) memcpy(work[i], data[i], n);
    for (unsigned i = mtrunc; i < m; i++) memset(work[i], 0, n);
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= m) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint16_t m01 = skew[iend], m02 = skew[iend + dist], m23 = skew[iend + 2 * dist];
            for (unsigned i = r; i < iend; i++) ifft4_16(work + i, dist, m01, m23, m02, n);
        }
        dist = dist4;
        dist4 <<= 2;
    }
    if (dist < m) {
        uint16_t lm = skew[dist];
        if (lm == L16_MOD)
            for (unsigned i = 0; i < dist; i++) xor_into(work[dist + i], work[i], n);
        else
            for (unsigned i = 0; i < dist; i++) ifft2_16(work[i], work[i + dist], lm, n);
    }
    if (xor_res)
        for (unsigned i = 0; i < m; i++) xor_into(xor_res[i], work[i], n);
}

/* leopard.go:650-693 ifftDITDecoder */
static void ifft_decoder16(unsigned mtrunc, uint8_t **work, unsigned m, const uint16_t *skew, size_t n) {
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= m) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint16_t m01 = skew[iend - 1], m02 = skew[iend + dist - 1], m23 = skew[iend + 2 * dist - 1];
            for (unsigned i = r; i < iend; i++) ifft4_16(work + i, dist, m01, m23, m02, n);
        }
        dist = dist4;
        dist4 <<= 2;
    }
    if (dist < m) {
        uint16_t lm = skew[dist - 1];
        if (lm == L16_MOD)
            for (unsigned i = 0; i < dist; i++) xor_into(work[dist + i], work[i], n);
        else
            for (unsigned i = 0; i < dist; i++) ifft2_16(work[i], work[i + dist], lm, n);
    }
}

/* leopard.go:696-736 fftDIT */
static void fft_dit16(uint8_t **work, unsigned mtrunc, unsigned m, const uint16_t *skew, size_t n) {
    unsigned dist4 = m, dist = m >> 2;
    while (dist != 0) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint16_t m01 = skew[iend - 1], m02 = skew[iend + dist - 1], m23 = skew[iend + 2 * dist - 1];
            for (unsigned i = r; i < iend; i++) fft4_16(work + i, dist, m01, m23, m02, n);
        }
        dist4 = dist;
        dist >>= 2;
    }
    if (dist4 == 2)
        for (unsigned r = 0; r < mtrunc; r += 2) {
            uint16_t lm = skew[r];
            if (lm == L16_MOD) xor_into(work[r + 1], work[r], n);
            else fft2_16(work[r], work[r + 1], lm, n);
        }
}

/* leopard.go:1017-1021 ceilPow2 */
static unsigned ceil_pow2(unsigned n) {
    unsigned r = 1;
    while (r < n) r <<= 1;
    return r;
}

static uint8_t **alloc_rows(unsigned count, size_t n) {
    uint8_t **w = (uint8_t **)malloc(sizeof(uint8_t *) * count);
    uint8_t *buf = (uint8_t *)calloc((size_t)count, n);
    for (unsigned i = 0; i < count; i++) w[i] = buf + (size_t)i * n;
    return w;
}
static void free_rows(uint8_t **w) {
    free(w[0]);
    free(w);
}

/* leopard.go:51-70 newFF16 argument checks */
static int leo16_check(int k, int p) {
    if (k <= 0 || p <= 0) return ORA_ERR_INV_SHARD_NUM;
    if (k + p > 65536) return ORA_ERR_MAX_SHARD_NUM;
    return ORA_OK;
}

/* leopard.go:169-270 encode + encodeChunk (whole shard as one chunk) */
int ora_leo16_encode(int k, int p, uint8_t *const *shards, size_t size) {
    int rc = leo16_check(k, p);
    if (rc) return rc;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    if (size % 64) return ORA_ERR_INVALID_SHARD_SIZE;
    leo16_init();
    unsigned m = ceil_pow2((unsigned)p), mtrunc = (unsigned)k < m ? (unsigned)k : m;
    unsigned last = (unsigned)k % m;
    uint8_t **scratch = alloc_rows(2 * m, size);
    uint8_t **work = (uint8_t **)malloc(sizeof(uint8_t *) * 2 * m);
    for (unsigned i = 0; i < 2 * m; i++) work[i] = i < (unsigned)p ? shards[k + i] : scratch[i];
    const uint16_t *skew = l16_skew + (m - 1);
    ifft_encoder16(shards, mtrunc, work, NULL, m, skew, size);
    if (m < (unsigned)k) {
        unsigned i = m;
        for (; i + m <= (unsigned)k; i += m) {
            skew += m;
            ifft_encoder16(shards + i, m, work + m, work, m, skew, size);
        }
        if (last) {
            skew += m;
            ifft_encoder16(shards + i, last, work + m, work, m, skew, size);
        }
    }
    fft_dit16(work, (unsigned)p, m, l16_skew, size);
    free(work);
    free_rows(scratch);
    return ORA_OK;
}

/* leopard.go:421-510 error locator evaluation */
int ora_leo16_errlocs(int k, int p, const uint8_t *present, uint16_t *errlocs_out) {
    leo16_init();
    unsigned m = ceil_pow2((unsigned)p);
    uint16_t *el = (uint16_t *)calloc(L16_ORDER, 2);
    for (int i = 0; i < p; i++)
        if (!present[k + i]) el[i] = 1;
    for (unsigned i = (unsigned)p; i < m; i++) el[i] = 1;
    for (int i = 0; i < k; i++)
        if (!present[i]) el[i + m] = 1;
    fwht16(el, m + (unsigned)k);
    for (unsigned i = 0; i < L16_ORDER; i++) el[i] = (uint16_t)(((unsigned)el[i] * l16_walsh[i]) % L16_MOD);
    fwht16(el, L16_ORDER);
    memcpy(errlocs_out, el, L16_ORDER * 2);
    free(el);
    return ORA_OK;
}

/* leopard.go:421-647 reconstruct + reconstructChunk (dense FFT; the errorBits
 * sparse FFT only skips outputs that are never revealed) */
int ora_leo16_reconstruct(int k, int p, uint8_t *const *shards, const uint8_t *present,
                          size_t size, int recover_all, uint8_t *written) {
    int rc = leo16_check(k, p);
    if (rc) return rc;
    int total = k + p, number_present = 0, data_present = 0;
    if (written) memset(written, 0, (size_t)total);
    for (int i = 0; i < total; i++)
        if (present[i]) { number_present++; if (i < k) data_present++; }
    if (number_present == 0 || size == 0) return ORA_ERR_SHARD_NO_DATA;
    if (number_present == total || (!recover_all && data_present == k)) return ORA_OK;
    if (number_present < k) return ORA_ERR_TOO_FEW_SHARDS;
    if (size % 64) return ORA_ERR_INVALID_SHARD_SIZE;
    leo16_init();
    unsigned m = ceil_pow2((unsigned)p), n = ceil_pow2(m + (unsigned)k);
    unsigned input_count = (unsigned)p;
    for (int i = 0; i < k; i++)
        if (present[i]) input_count = m + (unsigned)i + 1;
    uint16_t *el = (uint16_t *)malloc(L16_ORDER * 2);
    ora_leo16_errlocs(k, p, present, el);
    uint8_t **work = alloc_rows(n, size);
    for (int i = 0; i < p; i++)
        if (present[k + i]) mul16(work[i], shards[k + i], el[i], size);
    for (int i = 0; i < k; i++)
        if (present[i]) mul16(work[m + i], shards[i], el[m + i], size);
    ifft_decoder16(input_count, work, n, l16_skew, size);
    for (unsigned i = 1; i < n; i++) {
        unsigned width = ((i ^ (i - 1)) + 1) >> 1;
        for (unsigned j = 0; j < width; j++) xor_into(work[i - width + j], work[i + j], size);
    }
    fft_dit16(work, m + (unsigned)k, n, l16_skew, size);
    int end = recover_all ? total : k;
    for (int i = 0; i < end; i++) {
        if (present[i]) continue;
        if (i >= k) mul16(shards[i], work[i - k], (uint16_t)(L16_MOD - el[i - k]), size);
        else mul16(shards[i], work[i + m], (uint16_t)(L16_MOD - el[i + m]), size);
        if (written) written[i] = 1;
    }
    free_rows(work);
    free(el);
    return ORA_OK;
}

/* leopard.go:393-419 Verify */
int ora_leo16_verify(int k, int p, uint8_t *const *shards, size_t size, int *ok) {
    int rc = leo16_check(k, p);
    if (rc) return rc;
    uint8_t **outs = (uint8_t **)malloc(sizeof(uint8_t *) * (size_t)(k + p));
    uint8_t **par = alloc_rows((unsigned)p, size);
    for (int i = 0; i < k; i++) outs[i] = shards[i];
    for (int i = 0; i < p; i++) outs[k + i] = par[i];
    rc = ora_leo16_encode(k, p, outs, size);
    *ok = 1;
    for (int i = 0; rc == ORA_OK && i < p; i++)
        if (memcmp(par[i], shards[k + i], size)) *ok = 0;
    free_rows(par);
    free(outs);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Leopard GF(2^8) (leopard8.go)                                               */
/* ------------------------------------------------------------------------ */
#define L8_ORDER 256u
#define L8_MOD 255u
static uint8_t l8_log[256], l8_exp[256], l8_skew[255], l8_walsh[256];
static uint8_t l8_lut[256][256];
static int l8_ready;

static inline uint8_t add_mod8(uint8_t a, uint8_t b) {
    uint64_t s = (uint64_t)a + b;
    return (uint8_t)(s + (s >> 8));
}
static inline uint8_t sub_mod8(uint8_t a, uint8_t b) {
    uint64_t d = (uint64_t)a - (uint64_t)b;
    return (uint8_t)(d + (d >> 8));
}
/* leopard8.go:919-931 mulLog8 */
static inline uint8_t mullog8(uint8_t a, uint8_t log_b) {
    if (a == 0) return 0;
    return l8_exp[add_mod8(l8_log[a], log_b)];
}

/* leopard8.go:954-989 fwht8 */
static void fwht8(uint8_t *data, unsigned mtrunc) {
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= L8_ORDER) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            for (unsigned off = r; off < r + dist; off++) {
                uint8_t t0 = data[off], t1 = data[off + dist], t2 = data[off + 2 * dist], t3 = data[off + 3 * dist];
                uint8_t a, b;
                a = add_mod8(t0, t1); b = sub_mod8(t0, t1); t0 = a; t1 = b;
                a = add_mod8(t2, t3); b = sub_mod8(t2, t3); t2 = a; t3 = b;
                a = add_mod8(t0, t2); b = sub_mod8(t0, t2); t0 = a; t2 = b;
                a = add_mod8(t1, t3); b = sub_mod8(t1, t3); t1 = a; t3 = b;
                data[off] = t0; data[off + dist] = t1; data[off + 2 * dist] = t2; data[off + 3 * dist] = t3;
            }
        }
        dist = dist4;
        dist4 <<= 2;
    }
}

static void leo8_init(void) {
    if (l8_ready) return;
    static const uint8_t cantor[8] = {1, 214, 152, 146, 86, 200, 88, 230}; /* leopard8.go:1030-1032 */
    /* leopard8.go:1029-1071 initLUTs8 */
    unsigned state = 1;
    for (unsigned i = 0; i < L8_MOD; i++) {
        l8_exp[state] = (uint8_t)i;
        state <<= 1;
        if (state >= L8_ORDER) state ^= 0x11D;
    }
    l8_exp[0] = L8_MOD;
    l8_log[0] = 0;
    for (int i = 0; i < 8; i++) {
        unsigned width = 1u << i;
        for (unsigned j = 0; j < width; j++) l8_log[j + width] = l8_log[j] ^ cantor[i];
    }
    for (unsigned i = 0; i < L8_ORDER; i++) l8_log[i] = l8_exp[l8_log[i]];
    for (unsigned i = 0; i < L8_ORDER; i++) l8_exp[l8_log[i]] = (uint8_t)i;
    l8_exp[L8_MOD] = l8_exp[0];
    /* leopard8.go:1072-1117 initFFTSkew8 */
    uint8_t temp[7];
    memset(l8_skew, 0, sizeof l8_skew);
    for (int i = 1; i < 8; i++) temp[i - 1] = (uint8_t)(1u << i);
    for (int m = 0; m < 7; m++) {
        unsigned step = 1u << (m + 1);
        l8_skew[(1u << m) - 1] = 0;
        for (int i = m; i < 7; i++) {
            unsigned s = 1u << (i + 1);
            for (unsigned j = (1u << m) - 1; j < s; j += step) l8_skew[j + s] = l8_skew[j] ^ temp[i];
        }
        temp[m] = (uint8_t)(L8_MOD - l8_log[mullog8(temp[m], l8_log[temp[m] ^ 1])]);
        for (int i = m + 1; i < 7; i++) {
            uint8_t sum = add_mod8(l8_log[temp[i] ^ 1], temp[m]);
            temp[i] = mullog8(temp[i], sum);
        }
    }
    for (unsigned i = 0; i < L8_MOD; i++) l8_skew[i] = l8_log[l8_skew[i]];
    for (unsigned i = 0; i < L8_ORDER; i++) l8_walsh[i] = l8_log[i];
    l8_walsh[0] = 0;
    fwht8(l8_walsh, L8_ORDER);
    /* leopard8.go:1119-1137 initMul8LUT */
    for (unsigned lm = 0; lm < 256; lm++) {
        uint8_t tmp[32];
        for (int nib = 0, shift = 0; nib < 2; nib++, shift += 4)
            for (int x = 0; x < 16; x++) tmp[nib * 16 + x] = mullog8((uint8_t)(x << shift), (uint8_t)lm);
        for (int i = 0; i < 256; i++) l8_lut[lm][i] = tmp[i & 15] ^ tmp[(i >> 4) + 16];
    }
    l8_ready = 1;
}

void ora_leo8_tables(uint8_t *log_out, uint8_t *exp_out, uint8_t *skew_out, uint8_t *walsh_out) {
    leo8_init();
    if (log_out) memcpy(log_out, l8_log, 256);
    if (exp_out) memcpy(exp_out, l8_exp, 256);
    if (skew_out) memcpy(skew_out, l8_skew, 255);
    if (walsh_out) memcpy(walsh_out, l8_walsh, 256);
}

uint8_t ora_leo8_mullog(uint8_t a, uint8_t log_b) {
    leo8_init();
    return mullog8(a, log_b);
}

/* Bit matrix of x -> mulLog8(x, log_m) in the layout of leopard8.go:1271
 * gf2p811dMulMatricesLeo8 (same convention as leopard.go:1243-1254). */
uint64_t ora_leo8_gfni_matrix(uint8_t log_m) {
    leo8_init();
    uint64_t a = 0;
    for (int ib = 0; ib < 8; ib++) {
        uint8_t r = mullog8((uint8_t)(1u << ib), log_m);
        for (int ob = 0; ob < 8; ob++)
            if ((r >> ob) & 1) a |= (uint64_t)1 << ((7 - ob) * 8 + ib);
    }
    return a;
}

/* leopard8.go:891-916 refMulAdd8 / refMul8 */
static void muladd8(uint8_t *x, const uint8_t *y, uint8_t lm, size_t n) {
    const uint8_t *t = l8_lut[lm];
#if defined(__x86_64__) || defined(__i386__)
    if (leo_simd) {
        muladd8_avx2(x, y, t, n, 1);
        return;
    }
#endif
    for (size_t i = 0; i < n; i++) x[i] ^= t[y[i]];
}
static void mul8(uint8_t *x, const uint8_t *y, uint8_t lm, size_t n) {
    const uint8_t *t = l8_lut[lm];
#if defined(__x86_64__) || defined(__i386__)
    if (leo_simd) {
        muladd8_avx2(x, y, t, n, 0);
        return;
    }
#endif
    for (size_t i = 0; i < n; i++) x[i] = t[y[i]];
}
/* galois_noasm.go:101-105 fftDIT28, :115-119 ifftDIT28 */
static void fft2_8(uint8_t *x, uint8_t *y, uint8_t lm, size_t n) { muladd8(x, y, lm, n); xor_into(y, x, n); }
static void ifft2_8(uint8_t *x, uint8_t *y, uint8_t lm, size_t n) { xor_into(y, x, n); muladd8(x, y, lm, n); }

/* leopard8.go:726-749 fftDIT4Ref8 */
static void fft4_8(uint8_t **w, unsigned dist, uint8_t m01, uint8_t m23, uint8_t m02, size_t n) {
    if (m02 == L8_MOD) { xor_into(w[2 * dist], w[0], n); xor_into(w[3 * dist], w[dist], n); }
    else { fft2_8(w[0], w[2 * dist], m02, n); fft2_8(w[dist], w[3 * dist], m02, n); }
    if (m01 == L8_MOD) xor_into(w[dist], w[0], n); else fft2_8(w[0], w[dist], m01, n);
    if (m23 == L8_MOD) xor_into(w[3 * dist], w[2 * dist], n); else fft2_8(w[2 * dist], w[3 * dist], m23, n);
}
/* leopard8.go:858-880 ifftDIT4Ref8 */
static void ifft4_8(uint8_t **w, unsigned dist, uint8_t m01, uint8_t m23, uint8_t m02, size_t n) {
    if (m01 == L8_MOD) xor_into(w[dist], w[0], n); else ifft2_8(w[0], w[dist], m01, n);
    if (m23 == L8_MOD) xor_into(w[3 * dist], w[2 * dist], n); else ifft2_8(w[2 * dist], w[3 * dist], m23, n);
    if (m02 == L8_MOD) { xor_into(w[2 * dist], w[0], n); xor_into(w[3 * dist], w[dist], n); }
    else { ifft2_8(w[0], w[2 * dist], m02, n); ifft2_8(w[dist], w[3 * dist], m02, n); }
}

/* leopard8.go:755-856 ifftDITEncoder8 */
static void ifft_encoder8(uint8_t *const *data, unsigned mtrunc, uint8_t **work, uint8_t **xor_res,
                          unsigned m, const uint8_t *skew, size_t n) {
    for (unsigned i = 0; i < mtrunc; i++) memcpy(work[i], data[i], n);
    for (unsigned i = mtrunc; i < m; i++) memset(work[i], 0, n);
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= m) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint8_t m01 = skew[iend], m02 = skew[iend + dist], m23 = skew[iend + 2 * dist];
            for (unsigned i = r; i < iend; i++) ifft4_8(work + i, dist, m01, m23, m02, n);
        }
        dist = dist4;
        dist4 <<= 2;
    }
    if (dist < m) {
        uint8_t lm = skew[dist];
        if (lm == L8_MOD)
            for (unsigned i = 0; i < dist; i++) xor_into(work[dist + i], work[i], n);
        else
            for (unsigned i = 0; i < dist; i++) ifft2_8(work[i], work[i + dist], lm, n);
    }
    if (xor_res)
        for (unsigned i = 0; i < m; i++) xor_into(xor_res[i], work[i], n);
}

/* leopard8.go:637-680 ifftDITDecoder8 */
static void ifft_decoder8(unsigned mtrunc, uint8_t **work, unsigned m, const uint8_t *skew, size_t n) {
    unsigned dist = 1, dist4 = 4;
    while (dist4 <= m) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint8_t m01 = skew[iend - 1], m02 = skew[iend + dist - 1], m23 = skew[iend + 2 * dist - 1];
            for (unsigned i = r; i < iend; i++) ifft4_8(work + i, dist, m01, m23, m02, n);
        }
        dist = dist4;
        dist4 <<= 2;
    }
    if (dist < m) {
        uint8_t lm = skew[dist - 1];
        if (lm == L8_MOD)
            for (unsigned i = 0; i < dist; i++) xor_into(work[dist + i], work[i], n);
        else
            for (unsigned i = 0; i < dist; i++) ifft2_8(work[i], work[i + dist], lm, n);
    }
}

/* leopard8.go:683-723 fftDIT8 */
static void fft_dit8(uint8_t **work, unsigned mtrunc, unsigned m, const uint8_t *skew, size_t n) {
    unsigned dist4 = m, dist = m >> 2;
    while (dist != 0) {
        for (unsigned r = 0; r < mtrunc; r += dist4) {
            unsigned iend = r + dist;
            uint8_t m01 = skew[iend - 1], m02 = skew[iend + dist - 1], m23 = skew[iend + 2 * dist - 1];
            for (unsigned i = r; i < iend; i++) fft4_8(work + i, dist, m01, m23, m02, n);
        }
        dist4 = dist;
        dist >>= 2;
    }
    if (dist4 == 2)
        for (unsigned r = 0; r < mtrunc; r += 2) {
            uint8_t lm = skew[r];
            if (lm == L8_MOD) xor_into(work[r + 1], work[r], n);
            else fft2_8(work[r], work[r + 1], lm, n);
        }
}

/* leopard8.go:42-66 newFF8 checks.  The reference accepts ceilPow2(p)+k > 256
 * and then indexes past its 255-entry skew table (encode) and 256-entry
 * errLocs (reconstruct); that geometry is rejected here. */
static int leo8_check(int k, int p) {
    if (k <= 0 || p <= 0) return ORA_ERR_INV_SHARD_NUM;
    if (k + p > 65536) return ORA_ERR_MAX_SHARD_NUM;
    if (ceil_pow2((unsigned)p) + (unsigned)k > 256) return ORA_ERR_MAX_SHARD_NUM;
    return ORA_OK;
}

/* leopard8.go:139-243 encode */
int ora_leo8_encode(int k, int p, uint8_t *const *shards, size_t size) {
    int rc = leo8_check(k, p);
    if (rc) return rc;
    if (size == 0) return ORA_ERR_SHARD_NO_DATA;
    if (size % 64) return ORA_ERR_INVALID_SHARD_SIZE;
    leo8_init();
    unsigned m = ceil_pow2((unsigned)p), mtrunc = (unsigned)k < m ? (unsigned)k : m;
    unsigned last = (unsigned)k % m;
    uint8_t **scratch = alloc_rows(2 * m, size);
    uint8_t **work = (uint8_t **)malloc(sizeof(uint8_t *) * 2 * m);
    for (unsigned i = 0; i < 2 * m; i++) work[i] = i < (unsigned)p ? shards[k + i] : scratch[i];
    const uint8_t *skew = l8_skew + (m - 1);
    ifft_encoder8(shards, mtrunc, work, NULL, m, skew, size);
    if (m < (unsigned)k) {
        unsigned i = m;
        for (; i + m <= (unsigned)k; i += m) {
            skew += m;
            ifft_encoder8(shards + i, m, work + m, work, m, skew, size);
        }
        if (last) {
            skew += m;
            ifft_encoder8(shards + i, last, work + m, work, m, skew, size);
        }
    }
    fft_dit8(work, (unsigned)p, m, l8_skew, size);
    free(work);
    free_rows(scratch);
    return ORA_OK;
}

/* leopard8.go:430-513 error locator (the reference caches it per erasure set) */
int ora_leo8_errlocs(int k, int p, const uint8_t *present, uint8_t *errlocs_out) {
    leo8_init();
    unsigned m = ceil_pow2((unsigned)p);
    uint8_t el[256];
    memset(el, 0, sizeof el);
    for (int i = 0; i < p; i++)
        if (!present[k + i]) el[i] = 1;
    for (unsigned i = (unsigned)p; i < m; i++) el[i] = 1;
    for (int i = 0; i < k; i++)
        if (!present[i]) el[i + m] = 1;
    fwht8(el, m + (unsigned)k);
    for (unsigned i = 0; i < L8_ORDER; i++) el[i] = (uint8_t)(((unsigned)el[i] * l8_walsh[i]) % L8_MOD);
    fwht8(el, L8_ORDER);
    memcpy(errlocs_out, el, 256);
    return ORA_OK;
}

/* leopard8.go:393-634 reconstruct */
int ora_leo8_reconstruct(int k, int p, uint8_t *const *shards, const uint8_t *present,
                         size_t size, int recover_all, uint8_t *written) {
    int rc = leo8_check(k, p);
    if (rc) return rc;
    int total = k + p, number_present = 0, data_present = 0;
    if (written) memset(written, 0, (size_t)total);
    for (int i = 0; i < total; i++)
        if (present[i]) { number_present++; if (i < k) data_present++; }
    if (number_present == 0 || size == 0) return ORA_ERR_SHARD_NO_DATA;
    if (number_present == total || (!recover_all && data_present == k)) return ORA_OK;
    if (number_present < k) return ORA_ERR_TOO_FEW_SHARDS;
    if (size % 64) return ORA_ERR_INVALID_SHARD_SIZE;
    leo8_init();
    unsigned m = ceil_pow2((unsigned)p), n = ceil_pow2(m + (unsigned)k);
    uint8_t el[256];
    ora_leo8_errlocs(k, p, present, el);
    uint8_t **work = alloc_rows(n, size);
    for (int i = 0; i < p; i++)
        if (present[k + i]) mul8(work[i], shards[k + i], el[i], size);
    for (int i = 0; i < k; i++)
        if (present[i]) mul8(work[m + i], shards[i], el[m + i], size);
    ifft_decoder8(m + (unsigned)k, work, n, l8_skew, size);
    for (unsigned i = 1; i < n; i++) {
        unsigned width = ((i ^ (i - 1)) + 1) >> 1;
        for (unsigned j = 0; j < width; j++) xor_into(work[i - width + j], work[i + j], size);
    }
    fft_dit8(work, m + (unsigned)k, n, l8_skew, size);
    int end = recover_all ? total : k;
    for (int i = 0; i < end; i++) {
        if (present[i]) continue;
        if (i >= k) mul8(shards[i], work[i - k], (uint8_t)(L8_MOD - el[i - k]), size);
        else mul8(shards[i], work[i + m], (uint8_t)(L8_MOD - el[i + m]), size);
        if (written) written[i] = 1;
    }
    free_rows(work);
    return ORA_OK;
}

/* leopard8.go:365-391 Verify */
int ora_leo8_verify(int k, int p, uint8_t *const *shards, size_t size, int *ok) {
    int rc = leo8_check(k, p);
    if (rc) return rc;
    uint8_t **outs = (uint8_t **)malloc(sizeof(uint8_t *) * (size_t)(k + p));
    uint8_t **par = alloc_rows((unsigned)p, size);
    for (int i = 0; i < k; i++) outs[i] = shards[i];
    for (int i = 0; i < p; i++) outs[k + i] = par[i];
    rc = ora_leo8_encode(k, p, outs, size);
    *ok = 1;
    for (int i = 0; rc == ORA_OK && i < p; i++)
        if (memcmp(par[i], shards[k + i], size)) *ok = 0;
    free_rows(par);
    free(outs);
    return rc;
}
