// leopard.cu -- Leopard GF(2^16) / GF(2^8) FFT codec on sm_100a.
//
// Replaces leopardFF16.encode/reconstruct (leopard.go:169-647) and
// leopardFF8.encode/reconstruct (leopard8.go:139-634) and their SIMD
// butterflies (fftDIT4/ifftDIT4/fftDIT48/..., galois_amd64.go:206-1164).
//
// Every transform is column-local: one CTA owns a 64-byte column tile of
// every row (for GF(2^16) one chunk: 32 symbols as 32 low bytes | 32 high
// bytes, leopard.go:907-925; for GF(2^8) 64 byte symbols) and runs all
// butterfly layers of the encode (block IFFTs + XOR-accumulate + FFT) or the
// decode (scale, IFFT, formal derivative, FFT, reveal) in shared memory.  HBM
// is touched once per shard: algorithmic bytes = (k + p) * size for encode,
// (present + written) * size for decode.
//
// Multiplication by a constant log value lm uses split product tables
// (GF(2^16): 64 + 64 + 16 u16 per lm for symbol bits 0-5, 6-11, 12-15, 32 MB
// in global memory, L1/L2 resident, three lookups per symbol; GF(2^8):
// 2 x 16 bytes per lm, 8 KB in shared memory).  Each thread handles four
// symbols of a row per butterfly, and a warp's lanes share their
// multipliers once the butterfly distance reaches 4, so a lookup reads one
// 128-byte line per warp.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "leo_host.h"
#include "rsgpu_internal.h"

namespace rsgpu {

constexpr int kLeoThreads = 256;        // encode CTAs (2m rows of shared memory each)
constexpr int kLeoEncThreadsMax = 512;  // staged GF(2^16) encode: 2m threads up to this
constexpr int kLeoDecodeThreads = 1024; // decode CTAs hold up to 128 KB: one per SM, so 32 warps
constexpr int kLeoTile = 64;          // bytes of every row owned by one CTA
constexpr int kLeoMaxShards = 2048;   // shard pointers carried in kernel parameters
constexpr int kLeoMaxRows = 2048;     // rows held in shared memory (2048 * 64 B = 128 KB)

// Per-device tables (built once per context on first use).
struct LeoState {
    int device = -1;
    uint16_t *skew16 = nullptr;  // fftSkew, 65535 entries
    uint16_t *t16 = nullptr;     // [65536][kT16Stride] split product tables (see F16)
    uint16_t *ts16 = nullptr;    // [65535][4][16] nibble tables in fftSkew order (see F16S)
    uint16_t *tw16 = nullptr;    // [16384][128] wide tables of fftSkew indices 4j+3 (see F16W)
    uint16_t *skew8 = nullptr;   // fftSkew8, 255 entries (widened)
    uint8_t *t8 = nullptr;       // [256][2][16] nibble products
    uint16_t *fold16 = nullptr;  // W_n of FWHT(log) for n = 2^0..2^16 (see leo_errloc_kernel)
    uint16_t *fold8 = nullptr;   // W_n of FWHT(log8) for n = 2^0..2^8
    ~LeoState() {
        if (device >= 0) {
            cudaFree(skew16);
            cudaFree(t16);
            cudaFree(ts16);
            cudaFree(tw16);
            cudaFree(skew8);
            cudaFree(t8);
            cudaFree(fold16);
            cudaFree(fold8);
        }
    }
};

// Error locators per erasure pattern (the reference caches GF(2^8) ones,
// leopard8.go:465-513): device arrays of n entries keyed by the present-shard
// bitmask, each with an event recorded after the kernel that filled it, so a
// decode on any stream waits for it.  Entries are never evicted (a decode in
// flight may read any of them); past kErrLocCacheCap patterns the locators
// are computed per call.  Freed when the encoder is freed, after the device
// is idle.
struct LeoErrLocCache {
    int device = -1;
    std::mutex mu;
    struct Entry {
        uint16_t *d = nullptr;
        cudaEvent_t ready = nullptr;
    };
    std::map<std::vector<uint32_t>, Entry> map;
    ~LeoErrLocCache() {
        if (map.empty()) return;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaDeviceSynchronize();
        for (auto &kv : map) {
            cudaFree(kv.second.d);
            cudaEventDestroy(kv.second.ready);
        }
        cudaSetDevice(prev);
    }
};

int leo_errloc_cached(const rsgpu_encoder *enc) {
    if (!enc->errlocs) return 0;
    std::lock_guard<std::mutex> lk(enc->errlocs->mu);
    return (int)enc->errlocs->map.size();
}

namespace {

constexpr size_t kErrLocCacheCap = 256;
constexpr int kT16Stride = 256;  // u16 entries per log value (512 bytes, 4 L1 lines)

struct LeoEncArgs {
    const uint8_t *shard[kLeoMaxShards];  // k data then p parity pointers
    int k, p, m;
    long long size;
    const uint16_t *skew;
    const uint16_t *t16;
    const uint16_t *ts16;
    const uint16_t *tw16;
    const uint8_t *t8;
};

struct LeoDecArgs {
    const uint8_t *shard[kLeoMaxShards];
    const uint16_t *errloc;               // the first n error locators (device)
    const uint16_t *ts16;
    const uint16_t *tw16;
    uint32_t present[kLeoMaxShards / 32];
    uint32_t write[kLeoMaxShards / 32];   // missing shards to reveal
    int k, p, m, n, input_count;
    long long size;
    const uint16_t *skew;
    const uint16_t *t16;
    const uint8_t *t8;
};

__device__ __forceinline__ bool bit(const uint32_t *v, int i) { return (v[i >> 5] >> (i & 31)) & 1u; }

// ---- field policies -----------------------------------------------------
// A thread works on a "quad": 4 consecutive symbols of one 64-byte row tile.
// GF(2^16) rows hold 32 symbols as 32 low bytes | 32 high bytes
// (leopard.go:907-925), so a quad is the u32 word of low bytes at 4q and
// the word of high bytes at 32 + 4q; GF(2^8) rows hold 64 byte symbols, a
// quad is one u32 word.  Consecutive threads take consecutive quads of a
// row, so a warp covers 4 (GF(2^16)) or 2 (GF(2^8)) butterfly positions,
// which share their multipliers whenever the butterfly distance is >= 4.
struct F16 {
    static constexpr unsigned kMod = 65535;
    static constexpr int kQuads = 8;
    static constexpr int kQuadShift = 3;
    using Q = uint2;
    // Shared-memory rows interleave the words: quad c is (low word, high
    // word) at byte 8c, so a warp's 8-byte loads of consecutive rows are
    // contiguous.  Global rows keep the reference's 32 low | 32 high bytes.
    static __device__ __forceinline__ Q ld(const uint8_t *row, int q) { return reinterpret_cast<const uint2 *>(row)[q]; }
    static __device__ __forceinline__ void st(uint8_t *row, int q, Q v) { reinterpret_cast<uint2 *>(row)[q] = v; }
    static __device__ __forceinline__ Q ldg(const uint8_t *row, int q) {
        return make_uint2(__ldcs(reinterpret_cast<const uint32_t *>(row) + q),
                          __ldcs(reinterpret_cast<const uint32_t *>(row + 32) + q));
    }
    static __device__ __forceinline__ void stg(uint8_t *row, int q, Q v) {
        __stcs(reinterpret_cast<uint32_t *>(row) + q, v.x);
        __stcs(reinterpret_cast<uint32_t *>(row + 32) + q, v.y);
    }
    // Row tile copies between the two layouts, 16 bytes (4 quads) at a time;
    // part in [0, 2) selects quads 4*part .. 4*part+3.
    static __device__ __forceinline__ void row_in(uint8_t *row, const uint8_t *src, int part) {
        const uint4 lo = __ldcs(reinterpret_cast<const uint4 *>(src) + part);
        const uint4 hi = __ldcs(reinterpret_cast<const uint4 *>(src + 32) + part);
        reinterpret_cast<uint4 *>(row)[2 * part] = make_uint4(lo.x, hi.x, lo.y, hi.y);
        reinterpret_cast<uint4 *>(row)[2 * part + 1] = make_uint4(lo.z, hi.z, lo.w, hi.w);
    }
    static __device__ __forceinline__ void row_out(uint8_t *dst, const uint8_t *row, int part) {
        const uint4 a = reinterpret_cast<const uint4 *>(row)[2 * part];
        const uint4 b = reinterpret_cast<const uint4 *>(row)[2 * part + 1];
        __stcs(reinterpret_cast<uint4 *>(dst) + part, make_uint4(a.x, a.z, b.x, b.z));
        __stcs(reinterpret_cast<uint4 *>(dst + 32) + part, make_uint4(a.y, a.w, b.y, b.w));
    }
    static constexpr int kRowParts = 2;
    static __device__ __forceinline__ Q zero() { return make_uint2(0, 0); }
    static __device__ __forceinline__ void xor_into(Q &a, Q b) {
        a.x ^= b.x;
        a.y ^= b.y;
    }
    // Products by a log value lm split by symbol bits, in lm's 512-byte
    // slot: bytes [0,128) bits 0-5, [128,256) bits 6-11, [256,288) bits 12-15.
    // Each part fits one 128-byte line, so a warp whose lanes share lm reads
    // one line per lookup.  Byte offsets are assembled with one PRMT each:
    // the slot base has a zero low byte, and the low byte is 2 * index
    // (+128 for the middle part), prepared for four symbols at once.
    const uint16_t *t;
    const uint16_t *skew;
    // Butterfly multiplier by fftSkew index: the log value; the modulus
    // stands for a zero product and skips the multiply (galois_noasm.go:94-112).
    using C = uint32_t;
    __device__ __forceinline__ C coef(int idx) const { return skew[idx]; }
    __device__ __forceinline__ void mac(Q &x, Q y, C lm) const {
        if (lm != kMod) xor_into(x, mul(y, lm));
    }
    __device__ __forceinline__ Q mul(Q v, uint32_t lm) const {
        const char *T = reinterpret_cast<const char *>(t);
        const uint32_t base = lm << 9, base2 = base + 256;
        const uint32_t a0 = (v.x << 1) & 0x7E7E7E7Eu;
        const uint32_t a1 = ((v.x >> 5) & 0x06060606u) | ((v.y << 3) & 0x78787878u) | 0x80808080u;
        const uint32_t a2 = (v.y >> 3) & 0x1E1E1E1Eu;
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t sel = 0x7650u | (uint32_t)i;
            r[i] = (uint32_t)__ldg(reinterpret_cast<const uint16_t *>(T + __byte_perm(a0, base, sel))) ^
                   (uint32_t)__ldg(reinterpret_cast<const uint16_t *>(T + __byte_perm(a1, base, sel))) ^
                   (uint32_t)__ldg(reinterpret_cast<const uint16_t *>(T + __byte_perm(a2, base2, sel)));
        }
        const uint32_t r01 = __byte_perm(r[0], r[1], 0x5410), r23 = __byte_perm(r[2], r[3], 0x5410);
        return make_uint2(__byte_perm(r01, r23, 0x6420), __byte_perm(r01, r23, 0x7531));
    }
};

struct F8 {
    static constexpr unsigned kMod = 255;
    static constexpr int kQuads = 16;
    static constexpr int kQuadShift = 4;
    using Q = uint32_t;
    static __device__ __forceinline__ Q ld(const uint8_t *row, int q) { return reinterpret_cast<const uint32_t *>(row)[q]; }
    static __device__ __forceinline__ void st(uint8_t *row, int q, Q v) { reinterpret_cast<uint32_t *>(row)[q] = v; }
    static __device__ __forceinline__ Q ldg(const uint8_t *row, int q) {
        return __ldcs(reinterpret_cast<const uint32_t *>(row) + q);
    }
    static __device__ __forceinline__ void stg(uint8_t *row, int q, Q v) {
        __stcs(reinterpret_cast<uint32_t *>(row) + q, v);
    }
    static __device__ __forceinline__ void row_in(uint8_t *row, const uint8_t *src, int part) {
        reinterpret_cast<uint4 *>(row)[part] = __ldcs(reinterpret_cast<const uint4 *>(src) + part);
    }
    static __device__ __forceinline__ void row_out(uint8_t *dst, const uint8_t *row, int part) {
        __stcs(reinterpret_cast<uint4 *>(dst) + part, reinterpret_cast<const uint4 *>(row)[part]);
    }
    static constexpr int kRowParts = 4;
    static __device__ __forceinline__ Q zero() { return 0; }
    static __device__ __forceinline__ void xor_into(Q &a, Q b) { a ^= b; }
    // Shared copy of the 8 KB table, 256-byte aligned: [lm][lo nibble 16 |
    // hi nibble 16].  A lookup address is one PRMT of the prepared index
    // byte ((lm & 7) * 32 + 16 * high + nibble) into the 256-byte block of lm.
    uint32_t t;  // shared-space address
    const uint16_t *skew;
    using C = uint32_t;
    __device__ __forceinline__ C coef(int idx) const { return skew[idx]; }
    __device__ __forceinline__ void mac(Q &x, Q y, C lm) const {
        if (lm != kMod) xor_into(x, mul(y, lm));
    }
    __device__ __forceinline__ Q mul(Q v, uint32_t lm) const {
        const uint32_t blk = t + ((lm >> 3) << 8);
        const uint32_t slot = (lm & 7u) * 0x20202020u;
        const uint32_t lo = (v & 0x0F0F0F0Fu) | slot;
        const uint32_t hi = ((v >> 4) & 0x0F0F0F0Fu) | slot | 0x10101010u;
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t sel = 0x7650u | (uint32_t)i;
            uint32_t x, y;
            asm("ld.shared.u8 %0, [%1];" : "=r"(x) : "r"(__byte_perm(lo, blk, sel)));
            asm("ld.shared.u8 %0, [%1];" : "=r"(y) : "r"(__byte_perm(hi, blk, sel)));
            r[i] = x ^ y;
        }
        return __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
    }
};

// The table reads below are plain (non-volatile) inline-asm shared loads:
// their addresses derive from row data loaded after the barrier that ends
// staging, and their results feed row stores issued before the next barrier,
// so the compiler can schedule them freely but never across a barrier.
//
// GF(2^16) with the transform's multiplier tables staged in shared memory.
// A transform over fftSkew indices [lo, lo + count) stages, for slot
// s = index - lo, the four 16-entry nibble product tables of skew[index]
// (all zero when skew[index] is the modulus, which the reference treats as a
// zero product, so no test is needed).  Slot s lives at position t: t = s,
// or, when the transform never reads slots s = 3 (mod 4) from nibble tables
// (compact; see stage_skew_tables), t = 3 * (s >> 2) + (s & 3).  Position t
// is the 256-byte block t >> 1 at half (t & 1) * 128, with nibble table q at
// 32-byte position (q + group) & 3 of that half (group: s >> 2 for a
// contiguous transform), so the four groups a warp covers in a distance-1
// layer hit different banks.  A lookup address is one PRMT of a prepared
// index byte into the block base.
struct F16S : F16 {
    uint32_t tab;   // shared-space address of position 0 (256-byte aligned)
    uint32_t ctab;  // shared-space address of the per-position index bytes (4 B each)
    int lo;         // fftSkew index of slot 0
    using C = uint32_t;
    __device__ __forceinline__ C coef(int idx) const { return (uint32_t)(idx - lo); }
    static __device__ __forceinline__ uint32_t lds16(uint32_t addr) {
        uint32_t v;
        asm("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(addr));
        return v;
    }
    // Byte q of the position constant: the low address byte of nibble table q
    // of position t (sw: the slot's bank swizzle, its butterfly group).
    static __device__ __forceinline__ uint32_t pos_const(uint32_t t, uint32_t sw) {
        uint32_t c = 0;
#pragma unroll
        for (uint32_t q = 0; q < 4; q++) c |= (((t & 1u) << 7) | (((q + sw) & 3u) << 5)) << (8 * q);
        return c;
    }
    __device__ __forceinline__ void mac(Q &x, Q y, C t) const {
        const uint32_t base = tab + ((t >> 1) << 8);
        uint32_t k;
        asm("ld.shared.u32 %0, [%1];" : "=r"(k) : "r"(ctab + (t << 2)));
        // 2 * symbol bits 0-3, 4-7, 8-11, 12-15 with table q's byte in every lane
        const uint32_t n0 = ((y.x << 1) & 0x1E1E1E1Eu) | __byte_perm(k, 0, 0x0000);
        const uint32_t n1 = ((y.x >> 3) & 0x1E1E1E1Eu) | __byte_perm(k, 0, 0x1111);
        const uint32_t n2 = ((y.y << 1) & 0x1E1E1E1Eu) | __byte_perm(k, 0, 0x2222);
        const uint32_t n3 = ((y.y >> 3) & 0x1E1E1E1Eu) | __byte_perm(k, 0, 0x3333);
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t sel = 0x7650u | (uint32_t)i;
            r[i] = lds16(__byte_perm(n0, base, sel)) ^ lds16(__byte_perm(n1, base, sel)) ^
                   lds16(__byte_perm(n2, base, sel)) ^ lds16(__byte_perm(n3, base, sel));
        }
        const uint32_t r01 = __byte_perm(r[0], r[1], 0x5410), r23 = __byte_perm(r[2], r[3], 0x5410);
        x.x ^= __byte_perm(r01, r23, 0x6420);
        x.y ^= __byte_perm(r01, r23, 0x7531);
    }
};

// F16S over compact positions: slots = 3 (mod 4) are left out.
struct F16SC : F16S {
    __device__ __forceinline__ C coef(int idx) const {
        const uint32_t s = (uint32_t)(idx - lo);
        return 3 * (s >> 2) + (s & 3);
    }
};

// GF(2^16) products for butterfly layers of distance >= 4.  There the four
// butterfly positions a warp covers belong to one group and share its
// multiplier, so a warp's lookups all hit one table and a 64-entry table
// costs no bank conflicts: a product takes three lookups instead of four.
// Wide slot j (256 bytes, 256-byte aligned) holds, for one multiplier,
// mulLog(e, lm) for e < 64 at bytes [0, 128) (symbol bits 0-5),
// mulLog(e << 6, lm) for e < 32 at [128, 192) (bits 6-10) and
// mulLog(e << 11, lm) for e < 32 at [192, 256) (bits 11-15); all zero when
// lm is the modulus.  Those layers only use fftSkew indices = 3 (mod 4) (the
// distance is a multiple of 4 and group starts are multiples of 4 * dist),
// so the global source holds 16384 such tables, one per index 4j + 3.
struct F16W : F16 {
    uint32_t wtab;  // shared-space address of wide slot 0 (256-byte aligned)
    int lo;         // fftSkew index that maps to slot position 0 (see coef)
    using C = uint32_t;
    // Wide slot of fftSkew index idx: (idx - lo) >> 2, for idx - lo = 3 (mod 4).
    __device__ __forceinline__ C coef(int idx) const { return (uint32_t)(idx - lo) >> 2; }
    __device__ __forceinline__ void mac(Q &x, Q y, C j) const {
        const uint32_t base = wtab + (j << 8);
        const uint32_t a0 = (y.x << 1) & 0x7E7E7E7Eu;                                            // 2 * bits 0-5
        const uint32_t a1 = ((y.x >> 5) & 0x06060606u) | ((y.y << 3) & 0x38383838u) | 0x80808080u; // 128 + 2 * bits 6-10
        const uint32_t a2 = ((y.y >> 2) & 0x3E3E3E3Eu) | 0xC0C0C0C0u;                            // 192 + 2 * bits 11-15
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t sel = 0x7650u | (uint32_t)i;
            r[i] = F16S::lds16(__byte_perm(a0, base, sel)) ^ F16S::lds16(__byte_perm(a1, base, sel)) ^
                   F16S::lds16(__byte_perm(a2, base, sel));
        }
        const uint32_t r01 = __byte_perm(r[0], r[1], 0x5410), r23 = __byte_perm(r[2], r[3], 0x5410);
        x.x ^= __byte_perm(r01, r23, 0x6420);
        x.y ^= __byte_perm(r01, r23, 0x7531);
    }
};

// The field view a butterfly pass of distance >= 4 uses: the wide tables for
// the staged GF(2^16) transforms, the same field otherwise.
template <class F>
struct WideOf {
    using T = F;
    static __device__ __forceinline__ const F &get(const F &f, uint32_t) { return f; }
};
template <class FS>
struct WideOfStaged {
    using T = F16W;
    static __device__ __forceinline__ F16W get(const FS &f, uint32_t wtab) {
        F16W v;
        v.t = f.t;
        v.skew = f.skew;
        v.wtab = wtab;
        v.lo = f.lo;
        return v;
    }
};
template <>
struct WideOf<F16S> : WideOfStaged<F16S> {};
template <>
struct WideOf<F16SC> : WideOfStaged<F16SC> {};

// Copies the wide tables of `count` slots: slot j gets the table of fftSkew
// index index_of(j) (= 3 mod 4) from the global [16384][128] u16 source.
template <class IndexOf>
__device__ void stage_wide(uint8_t *wtab, const uint16_t *tw16, unsigned count, IndexOf index_of) {
    for (unsigned v = threadIdx.x; v < count * 16; v += blockDim.x) {
        const unsigned j = v >> 4, part = v & 15;
        reinterpret_cast<uint4 *>(wtab + (size_t)j * 256)[part] =
            __ldg(reinterpret_cast<const uint4 *>(tw16 + (size_t)(index_of(j) >> 2) * 128) + part);
    }
}

// Copies nibble tables from the skew-ordered global table ([65535][4][16]
// u16) into positions [0, count) of the F16S layout, and writes each
// position's index bytes to ctab.  index_of(t): the fftSkew index staged at
// position t; swizzle_of(t): its bank swizzle, which must differ between the
// (up to four) butterfly groups one warp covers in a layer with distance 1.
template <class IndexOf, class SwizzleOf>
__device__ void stage_slots(uint8_t *tab, uint32_t *ctab, const uint16_t *ts16, unsigned count, IndexOf index_of,
                            SwizzleOf swizzle_of) {
    for (unsigned v = threadIdx.x; v < count * 8; v += blockDim.x) {
        const unsigned t = v >> 3, q = (v >> 1) & 3, h = v & 1;
        const uint4 x = __ldg(reinterpret_cast<const uint4 *>(ts16 + (size_t)index_of(t) * 64 + q * 16) + h);
        *reinterpret_cast<uint4 *>(tab + (t >> 1) * 256 + (t & 1) * 128 + ((q + swizzle_of(t)) & 3) * 32 + h * 16) = x;
    }
    for (unsigned t = threadIdx.x; t < count; t += blockDim.x) ctab[t] = F16S::pos_const(t, swizzle_of(t));
}

// Nibble positions of a contiguous transform of count slots: all of them, or
// (compact) those of slots s != 3 (mod 4).
__device__ __forceinline__ unsigned nibble_positions(unsigned count, bool compact) {
    return compact ? count - count / 4 : count;
}

// Contiguous fftSkew indices: slot s = index - lo; group of slot s is s >> 2.
// With wide tables (wtab != nullptr, lo a multiple of 4) the slots s = 3
// (mod 4) also go to wide slot s >> 2 for the layers of distance >= 4.  The
// only other readers of those slots are distance-2 passes (an FFT over
// 2^odd rows: slots r+1, r+3, r+5 of groups r = 0 mod 8); a transform
// without one stages them only as wide tables (compact positions, F16S).
__device__ void stage_skew_tables(uint8_t *tab, uint32_t *ctab, const uint16_t *ts16, int lo, int count,
                                  bool compact, uint8_t *wtab = nullptr, const uint16_t *tw16 = nullptr) {
    const unsigned npos = nibble_positions((unsigned)count, compact);
    if (compact)
        stage_slots(tab, ctab, ts16, npos, [lo](unsigned t) { return (unsigned)lo + 4 * (t / 3) + t % 3; },
                    [](unsigned t) { return t / 3; });
    else
        stage_slots(tab, ctab, ts16, npos, [lo](unsigned s) { return (unsigned)lo + s; },
                    [](unsigned s) { return s >> 2; });
    if (wtab) stage_wide(wtab, tw16, (unsigned)count / 4, [lo](unsigned j) { return (unsigned)lo + 4 * j + 3; });
}

// Butterflies (galois_noasm.go:94-112; a log multiplier equal to the modulus
// stands for multiplication by zero and reduces the butterfly to an XOR).
template <class F>
__device__ __forceinline__ void fft2(const F &f, typename F::Q &x, typename F::Q &y, typename F::C c) {
    f.mac(x, y, c);
    F::xor_into(y, x);
}
template <class F>
__device__ __forceinline__ void ifft2(const F &f, typename F::Q &x, typename F::Q &y, typename F::C c) {
    F::xor_into(y, x);
    f.mac(x, y, c);
}

// One radix-4 pass of the IFFT with decimation in time (ifftDITEncoder
// leopard.go:764-873 with skew_off = m-1+block*m, ifftDITDecoder :650-693
// with skew_off = -1): layers dist and 2*dist, multipliers
// skew[skew_off + iend], [+dist], [+2*dist]; groups start below mtrunc.
template <class F>
__device__ void ifft_pass4(const F &f, uint8_t *w, unsigned mtrunc, unsigned dist, unsigned ld, int skew_off) {
    using Q = typename F::Q;
    const unsigned groups = (mtrunc + (dist << 2) - 1) >> (ld + 2);
    const unsigned items = (groups << ld) << F::kQuadShift;
    for (unsigned it = threadIdx.x; it < items; it += blockDim.x) {
        const unsigned q = it >> F::kQuadShift, c = it & (F::kQuads - 1);
        const unsigned r = (q >> ld) << (ld + 2), i = r + (q & (dist - 1)), iend = r + dist;
        const typename F::C m01 = f.coef(skew_off + (int)iend);
        const typename F::C m02 = f.coef(skew_off + (int)(iend + dist));
        const typename F::C m23 = f.coef(skew_off + (int)(iend + 2 * dist));
        uint8_t *p0 = w + (size_t)i * kLeoTile;
        uint8_t *p1 = p0 + (size_t)dist * kLeoTile, *p2 = p1 + (size_t)dist * kLeoTile,
                *p3 = p2 + (size_t)dist * kLeoTile;
        Q x0 = F::ld(p0, c), x1 = F::ld(p1, c), x2 = F::ld(p2, c), x3 = F::ld(p3, c);
        ifft2(f, x0, x1, m01);
        ifft2(f, x2, x3, m23);
        ifft2(f, x0, x2, m02);
        ifft2(f, x1, x3, m02);
        F::st(p0, c, x0);
        F::st(p1, c, x1);
        F::st(p2, c, x2);
        F::st(p3, c, x3);
    }
    __syncthreads();
}

// The radix-2 IFFT layer left when log2(m) is odd (dist == m / 2).
template <class F>
__device__ void ifft_pass2(const F &f, uint8_t *w, unsigned dist, int skew_off) {
    using Q = typename F::Q;
    const typename F::C lm = f.coef(skew_off + (int)dist);
    const unsigned items = dist << F::kQuadShift;
    for (unsigned it = threadIdx.x; it < items; it += blockDim.x) {
        const unsigned i = it >> F::kQuadShift, c = it & (F::kQuads - 1);
        uint8_t *p0 = w + (size_t)i * kLeoTile, *p1 = p0 + (size_t)dist * kLeoTile;
        Q x = F::ld(p0, c), y = F::ld(p1, c);
        ifft2(f, x, y, lm);
        F::st(p0, c, x);
        F::st(p1, c, y);
    }
    __syncthreads();
}

// IFFT over m rows.  Passes of distance >= 4 use the field's wide view
// (WideOf; wtab: shared address of the wide slots, staged GF(2^16) only).
template <class F>
__device__ void ifft_rows(const F &f, uint8_t *w, unsigned mtrunc, unsigned m, int skew_off, uint32_t wtab = 0) {
    unsigned dist = 1, dist4 = 4, ld = 0;  // dist == 1 << ld
    for (; dist4 <= m; dist = dist4, dist4 <<= 2, ld += 2) {
        if (dist >= 4) ifft_pass4(WideOf<F>::get(f, wtab), w, mtrunc, dist, ld, skew_off);
        else ifft_pass4(f, w, mtrunc, dist, ld, skew_off);
    }
    if (dist < m) {  // one radix-2 layer left (dist == m / 2)
        if (dist >= 4) ifft_pass2(WideOf<F>::get(f, wtab), w, dist, skew_off);
        else ifft_pass2(f, w, dist, skew_off);
    }
}

// One radix-4 pass of the FFT with decimation in time (fftDIT
// leopard.go:696-736): multipliers skew[iend-1], [iend+dist-1],
// [iend+2*dist-1]; groups start below mtrunc.
template <class F>
__device__ void fft_pass4(const F &f, uint8_t *w, unsigned mtrunc, unsigned dist, unsigned ld) {
    using Q = typename F::Q;
    const unsigned groups = (mtrunc + (dist << 2) - 1) >> (ld + 2);
    const unsigned items = (groups << ld) << F::kQuadShift;
    for (unsigned it = threadIdx.x; it < items; it += blockDim.x) {
        const unsigned q = it >> F::kQuadShift, c = it & (F::kQuads - 1);
        const unsigned r = (q >> ld) << (ld + 2), i = r + (q & (dist - 1)), iend = r + dist;
        const typename F::C m01 = f.coef((int)iend - 1), m02 = f.coef((int)(iend + dist) - 1),
                            m23 = f.coef((int)(iend + 2 * dist) - 1);
        uint8_t *p0 = w + (size_t)i * kLeoTile;
        uint8_t *p1 = p0 + (size_t)dist * kLeoTile, *p2 = p1 + (size_t)dist * kLeoTile,
                *p3 = p2 + (size_t)dist * kLeoTile;
        Q x0 = F::ld(p0, c), x1 = F::ld(p1, c), x2 = F::ld(p2, c), x3 = F::ld(p3, c);
        fft2(f, x0, x2, m02);
        fft2(f, x1, x3, m02);
        fft2(f, x0, x1, m01);
        fft2(f, x2, x3, m23);
        F::st(p0, c, x0);
        F::st(p1, c, x1);
        F::st(p2, c, x2);
        F::st(p3, c, x3);
    }
    __syncthreads();
}

// FFT over m rows; passes of distance >= 4 use the wide view (see ifft_rows).
template <class F>
__device__ void fft_rows(const F &f, uint8_t *w, unsigned mtrunc, unsigned m, uint32_t wtab = 0) {
    using Q = typename F::Q;
    unsigned dist4 = m, dist = m >> 2;
    unsigned ld = 0;  // dist == 1 << ld
    while ((2u << ld) <= dist) ld++;
    for (; dist != 0; dist4 = dist, dist >>= 2, ld -= 2) {
        if (dist >= 4) fft_pass4(WideOf<F>::get(f, wtab), w, mtrunc, dist, ld);
        else fft_pass4(f, w, mtrunc, dist, ld);
    }
    if (dist4 == 2) {
        const unsigned items = ((mtrunc + 1) / 2) << F::kQuadShift;
        for (unsigned it = threadIdx.x; it < items; it += blockDim.x) {
            const unsigned r = 2 * (it >> F::kQuadShift), c = it & (F::kQuads - 1);
            const typename F::C lm = f.coef((int)r);
            uint8_t *p0 = w + (size_t)r * kLeoTile, *p1 = p0 + kLeoTile;
            Q x = F::ld(p0, c), y = F::ld(p1, c);
            fft2(f, x, y, lm);
            F::st(p0, c, x);
            F::st(p1, c, y);
        }
        __syncthreads();
    }
}

// Copies rows [first, first+cnt) of the shard list into w rows [0, cnt)
// (in the field's shared-memory layout) and zero-fills rows [cnt, rows).
template <class F>
__device__ void load_rows(uint8_t *w, const uint8_t *const *shard, int first, int cnt, int rows, long long off) {
    for (int v = threadIdx.x; v < rows * F::kRowParts; v += blockDim.x) {
        const int r = v / F::kRowParts, c = v % F::kRowParts;
        uint8_t *row = w + (size_t)r * kLeoTile;
        if (r < cnt) {
            F::row_in(row, shard[first + r] + off, c);
        } else {
            constexpr int kVecs = 4 / F::kRowParts;  // 16-byte vectors per part
#pragma unroll
            for (int j = 0; j < kVecs; j++) reinterpret_cast<uint4 *>(row)[c * kVecs + j] = make_uint4(0, 0, 0, 0);
        }
    }
}

template <class F>
__device__ void load_tables8(uint8_t *dst, const uint8_t *src) {
    for (int i = threadIdx.x; i < 256 * 32 / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
}

template <class F>
__device__ __forceinline__ F make_field(const uint16_t *t16, uint8_t *t8_shared, const uint16_t *skew);
template <>
__device__ __forceinline__ F16 make_field<F16>(const uint16_t *t16, uint8_t *, const uint16_t *skew) {
    F16 f;
    f.t = t16;
    f.skew = skew;
    return f;
}
template <>
__device__ __forceinline__ F8 make_field<F8>(const uint16_t *, uint8_t *t8s, const uint16_t *skew) {
    F8 f;
    f.t = (uint32_t)__cvta_generic_to_shared(t8s);
    f.skew = skew;
    return f;
}

constexpr int kT8Bytes = 256 * 32;
constexpr int kT8Slack = 256;  // the shared table starts at the next 256-byte boundary

__device__ __forceinline__ uint8_t *align_shared256(uint8_t *p) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(p);
    return p + ((256u - (s & 255u)) & 255u);
}

// Encode: IFFT of each m-row data block into tmp, XOR-accumulated into acc,
// then FFT of acc; rows [0, p) of acc are the parity (leopard.go:216-270).
template <class F>
__global__ void __launch_bounds__(kLeoThreads) leo_encode_kernel(const __grid_constant__ LeoEncArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    const bool gf8 = F::kQuads == 16;
    uint8_t *t8 = gf8 ? align_shared256(sm) : sm;
    uint8_t *acc = gf8 ? t8 + kT8Bytes : sm;
    const unsigned m = (unsigned)a.m;
    uint8_t *tmp = acc + (size_t)m * kLeoTile;
    if (gf8) load_tables8<F>(t8, a.t8);
    const F f = make_field<F>(a.t16, t8, a.skew);
    const long long off = (long long)blockIdx.x * kLeoTile;
    const int cnt0 = a.k < (int)m ? a.k : (int)m;
    load_rows<F>(acc, a.shard, 0, cnt0, (int)m, off);
    __syncthreads();
    ifft_rows(f, acc, (unsigned)cnt0, m, (int)m - 1);
    for (int b = 1; b * (int)m < a.k; b++) {
        const int start = b * (int)m;
        const int cnt = a.k - start < (int)m ? a.k - start : (int)m;
        load_rows<F>(tmp, a.shard, start, cnt, (int)m, off);
        __syncthreads();
        ifft_rows(f, tmp, (unsigned)cnt, m, (int)m - 1 + b * (int)m);
        for (int v = threadIdx.x; v < (int)m * 4; v += blockDim.x)
            reinterpret_cast<uint4 *>(acc)[v] = make_uint4(
                reinterpret_cast<uint4 *>(acc)[v].x ^ reinterpret_cast<uint4 *>(tmp)[v].x,
                reinterpret_cast<uint4 *>(acc)[v].y ^ reinterpret_cast<uint4 *>(tmp)[v].y,
                reinterpret_cast<uint4 *>(acc)[v].z ^ reinterpret_cast<uint4 *>(tmp)[v].z,
                reinterpret_cast<uint4 *>(acc)[v].w ^ reinterpret_cast<uint4 *>(tmp)[v].w);
        __syncthreads();
    }
    fft_rows(f, acc, (unsigned)a.p, m);
    for (int v = threadIdx.x; v < a.p * F::kRowParts; v += blockDim.x) {
        const int r = v / F::kRowParts, c = v % F::kRowParts;
        F::row_out(const_cast<uint8_t *>(a.shard[a.k + r]) + off, acc + (size_t)r * kLeoTile, c);
    }
}

// Shared layout of the staged GF(2^16) encode for m rows per block: 2m data
// rows, the nibble positions (256-byte blocks of two), the wide slots of the
// indices = 3 (mod 4), the 4-byte position constants.  The IFFTs never read
// slots = 3 (mod 4) from nibble tables, nor does an FFT over 2^even rows;
// an FFT over 2^odd rows has a distance-2 pass that does, so m = 2^odd keeps
// every nibble position.
struct EncLayout {
    unsigned rows_bytes, nib_pos, wide, tab_bytes, wide_bytes;
    __host__ __device__ explicit EncLayout(unsigned m) {
        const unsigned count = m - 1;
        const bool odd = log2u(m) & 1;
        rows_bytes = 2 * m * kLeoTile;
        nib_pos = odd ? count : count - count / 4;
        wide = count / 4;
        tab_bytes = (nib_pos + 1) / 2 * 256;
        wide_bytes = wide * 256;
    }
    __host__ __device__ static unsigned log2u(unsigned v) {  // v a power of two
        unsigned n = 0;
        while (v > 1) {
            v >>= 1;
            n++;
        }
        return n;
    }
    __host__ __device__ size_t bytes() const { return (size_t)rows_bytes + tab_bytes + wide_bytes + nib_pos * 4 + 256; }
};

// GF(2^16) encode with each transform's multiplier tables staged in shared
// memory (F16S nibble positions for the distance-1 and -2 passes, F16W wide
// slots for the passes of distance >= 4; EncLayout), used while that fits one
// CTA (m <= 512).  Block size: 2m threads up to 512, one butterfly quad per
// thread in a radix-4 pass; at m = 256, 74.5 KB and 40 registers, so three
// CTAs per SM.
__global__ void __launch_bounds__(kLeoEncThreadsMax) leo_encode16_staged_kernel(const __grid_constant__ LeoEncArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    const unsigned m = (unsigned)a.m;
    const EncLayout L(m);
    uint8_t *acc = sm, *tmp = sm + (size_t)m * kLeoTile;
    uint8_t *tab = align_shared256(tmp + (size_t)m * kLeoTile);
    uint8_t *wtab = tab + L.tab_bytes;
    uint32_t *ctab = reinterpret_cast<uint32_t *>(wtab + L.wide_bytes);
    const uint32_t wtab_s = (uint32_t)__cvta_generic_to_shared(wtab);
    const bool fft_compact = L.nib_pos != m - 1;
    F16SC f;  // the IFFTs use compact positions
    f.t = a.t16;
    f.skew = a.skew;
    f.tab = (uint32_t)__cvta_generic_to_shared(tab);
    f.ctab = (uint32_t)__cvta_generic_to_shared(ctab);
    const long long off = (long long)blockIdx.x * kLeoTile;
    const int cnt0 = a.k < (int)m ? a.k : (int)m;
    load_rows<F16>(acc, a.shard, 0, cnt0, (int)m, off);
    f.lo = (int)m;  // block 0 reads fftSkew[m .. 2m-2]
    stage_skew_tables(tab, ctab, a.ts16, f.lo, (int)m - 1, true, wtab, a.tw16);
    __syncthreads();
    ifft_rows(f, acc, (unsigned)cnt0, m, (int)m - 1, wtab_s);
    for (int b = 1; b * (int)m < a.k; b++) {
        const int start = b * (int)m;
        const int cnt = a.k - start < (int)m ? a.k - start : (int)m;
        load_rows<F16>(tmp, a.shard, start, cnt, (int)m, off);
        f.lo = (int)m + b * (int)m;
        stage_skew_tables(tab, ctab, a.ts16, f.lo, (int)m - 1, true, wtab, a.tw16);
        __syncthreads();
        ifft_rows(f, tmp, (unsigned)cnt, m, (int)m - 1 + b * (int)m, wtab_s);
        for (int v = threadIdx.x; v < (int)m * 4; v += blockDim.x) {
            uint4 x = reinterpret_cast<uint4 *>(acc)[v];
            const uint4 y = reinterpret_cast<const uint4 *>(tmp)[v];
            x.x ^= y.x;
            x.y ^= y.y;
            x.z ^= y.z;
            x.w ^= y.w;
            reinterpret_cast<uint4 *>(acc)[v] = x;
        }
        __syncthreads();
    }
    f.lo = 0;  // the FFT reads fftSkew[0 .. m-2]
    stage_skew_tables(tab, ctab, a.ts16, 0, (int)m - 1, fft_compact, wtab, a.tw16);
    __syncthreads();
    if (fft_compact) fft_rows(f, acc, (unsigned)a.p, m, wtab_s);
    else fft_rows(static_cast<const F16S &>(f), acc, (unsigned)a.p, m, wtab_s);
    for (int v = threadIdx.x; v < a.p * F16::kRowParts; v += blockDim.x) {
        const int r = v / F16::kRowParts, c = v % F16::kRowParts;
        F16::row_out(const_cast<uint8_t *>(a.shard[a.k + r]) + off, acc + (size_t)r * kLeoTile, c);
    }
}

// ---- GF(2^16) decode with staged tables ---------------------------------
// The decode transforms span n <= 2048 rows, whose n-1 multipliers do not fit
// next to the 128 KB of rows, so each layer is staged in chunks of groups:
// slot 3*(g - g0) + t holds fftSkew[4*dist*g + (t+1)*dist - 1], the t-th
// multiplier (m01, m02, m23) of group g (ifftDITDecoder / fftDIT index them
// identically, leopard.go:650-736).
__device__ void formal_derivative(uint8_t *w, unsigned n);

constexpr unsigned kDecChunkSlots = 672;
constexpr size_t kDecTableBytes = 98304;  // >= kDecChunkSlots / 2 * 256 + kDecChunkSlots * 4
constexpr unsigned kDecWideSlots = kDecTableBytes / 256;  // 128 groups of 3 wide slots
static_assert((size_t)kDecChunkSlots / 2 * 256 + (size_t)kDecChunkSlots * 4 <= kDecTableBytes, "nibble chunk");

// The butterflies of groups g0 .. g0+cnt-1 of one radix-4 pass whose
// multipliers sit in slots 3*(g - g0) + (0: m01, 1: m02, 2: m23) of the
// field view f (nibble slots for distances 1 and 2, wide ones from 4).
template <bool kFft, class FV>
__device__ void radix4_chunk(const FV &f, uint8_t *w, unsigned g0, unsigned cnt, unsigned dist, unsigned ld) {
    using Q = F16::Q;
    const unsigned items = (cnt << ld) << F16::kQuadShift;
    for (unsigned it = threadIdx.x; it < items; it += blockDim.x) {
        const unsigned q = it >> F16::kQuadShift, c = it & (F16::kQuads - 1);
        const unsigned gl = q >> ld;
        const unsigned r = (g0 + gl) << (ld + 2), i = r + (q & (dist - 1));
        const uint32_t s01 = gl * 3, s02 = s01 + 1, s23 = s01 + 2;
        uint8_t *p0 = w + (size_t)i * kLeoTile;
        uint8_t *p1 = p0 + (size_t)dist * kLeoTile, *p2 = p1 + (size_t)dist * kLeoTile,
                *p3 = p2 + (size_t)dist * kLeoTile;
        Q x0 = F16::ld(p0, c), x1 = F16::ld(p1, c), x2 = F16::ld(p2, c), x3 = F16::ld(p3, c);
        if (kFft) {
            fft2(f, x0, x2, s02);
            fft2(f, x1, x3, s02);
            fft2(f, x0, x1, s01);
            fft2(f, x2, x3, s23);
        } else {
            ifft2(f, x0, x1, s01);
            ifft2(f, x2, x3, s23);
            ifft2(f, x0, x2, s02);
            ifft2(f, x1, x3, s02);
        }
        F16::st(p0, c, x0);
        F16::st(p1, c, x1);
        F16::st(p2, c, x2);
        F16::st(p3, c, x3);
    }
    __syncthreads();
}

// Slot t of group g holds fftSkew[4*dist*g + (t+1)*dist - 1].  From distance
// 4 on those indices are = 3 (mod 4) and the wide tables are staged instead,
// up to 128 groups per chunk.
template <bool kFft>
__device__ void radix4_staged(const F16S &f, uint8_t *w, uint8_t *tab, uint32_t *ctab, const uint16_t *ts16,
                              const uint16_t *tw16, unsigned mtrunc, unsigned dist, unsigned ld) {
    const unsigned groups = (mtrunc + (dist << 2) - 1) >> (ld + 2);
    const auto index_of = [=](unsigned g0) {
        return [=](unsigned s) { return 4 * dist * (g0 + s / 3) + (s % 3 + 1) * dist - 1; };
    };
    if (dist >= 4) {
        const F16W fw = WideOf<F16S>::get(f, (uint32_t)__cvta_generic_to_shared(tab));
        constexpr unsigned kPer = kDecWideSlots / 3;
        for (unsigned g0 = 0; g0 < groups; g0 += kPer) {
            const unsigned cnt = groups - g0 < kPer ? groups - g0 : kPer;
            stage_wide(tab, tw16, cnt * 3, index_of(g0));
            __syncthreads();
            radix4_chunk<kFft>(fw, w, g0, cnt, dist, ld);
        }
        return;
    }
    constexpr unsigned kPer = kDecChunkSlots / 3;
    for (unsigned g0 = 0; g0 < groups; g0 += kPer) {
        const unsigned cnt = groups - g0 < kPer ? groups - g0 : kPer;
        stage_slots(tab, ctab, ts16, cnt * 3, index_of(g0), [](unsigned s) { return s / 3; });
        __syncthreads();
        radix4_chunk<kFft>(f, w, g0, cnt, dist, ld);
    }
}

// ifftDITDecoder (leopard.go:650-693) over n rows, groups below mtrunc.
__device__ void ifft_staged(const F16S &f, uint8_t *w, uint8_t *tab, uint32_t *ctab, const uint16_t *ts16,
                            const uint16_t *tw16, unsigned mtrunc, unsigned n) {
    unsigned dist = 1, dist4 = 4, ld = 0;
    for (; dist4 <= n; dist = dist4, dist4 <<= 2, ld += 2)
        radix4_staged<false>(f, w, tab, ctab, ts16, tw16, mtrunc, dist, ld);
    if (dist < n) {  // one radix-2 layer left (dist == n / 2): multiplier fftSkew[dist - 1]
        auto layer = [&](const auto &fv) {
            for (unsigned it = threadIdx.x; it < (dist << F16::kQuadShift); it += blockDim.x) {
                const unsigned i = it >> F16::kQuadShift, c = it & (F16::kQuads - 1);
                uint8_t *p0 = w + (size_t)i * kLeoTile, *p1 = p0 + (size_t)dist * kLeoTile;
                F16::Q x = F16::ld(p0, c), y = F16::ld(p1, c);
                ifft2(fv, x, y, 0u);
                F16::st(p0, c, x);
                F16::st(p1, c, y);
            }
            __syncthreads();
        };
        if (dist >= 4) {
            stage_wide(tab, tw16, 1, [=](unsigned) { return dist - 1; });
            __syncthreads();
            layer(WideOf<F16S>::get(f, (uint32_t)__cvta_generic_to_shared(tab)));
        } else {
            stage_slots(tab, ctab, ts16, 1, [=](unsigned) { return dist - 1; }, [](unsigned) { return 0u; });
            __syncthreads();
            layer(f);
        }
    }
}

// fftDIT (leopard.go:696-736) over n rows, groups below mtrunc.
__device__ void fft_staged(const F16S &f, uint8_t *w, uint8_t *tab, uint32_t *ctab, const uint16_t *ts16,
                           const uint16_t *tw16, unsigned mtrunc, unsigned n) {
    unsigned dist4 = n, dist = n >> 2, ld = 0;
    while ((2u << ld) <= dist) ld++;
    for (; dist != 0; dist4 = dist, dist >>= 2, ld -= 2)
        radix4_staged<true>(f, w, tab, ctab, ts16, tw16, mtrunc, dist, ld);
    if (dist4 == 2) {  // final radix-2 layer: pair (r, r+1) multiplied by fftSkew[r]
        const unsigned pairs = (mtrunc + 1) / 2;
        for (unsigned p0 = 0; p0 < pairs; p0 += kDecChunkSlots) {
            const unsigned cnt = pairs - p0 < kDecChunkSlots ? pairs - p0 : kDecChunkSlots;
            stage_slots(tab, ctab, ts16, cnt, [=](unsigned s) { return 2 * (p0 + s); }, [](unsigned s) { return s; });
            __syncthreads();
            for (unsigned it = threadIdx.x; it < (cnt << F16::kQuadShift); it += blockDim.x) {
                const unsigned sl = it >> F16::kQuadShift, c = it & (F16::kQuads - 1);
                uint8_t *q0 = w + (size_t)(2 * (p0 + sl)) * kLeoTile, *q1 = q0 + kLeoTile;
                F16::Q x = F16::ld(q0, c), y = F16::ld(q1, c);
                fft2(f, x, y, sl);
                F16::st(q0, c, x);
                F16::st(q1, c, y);
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kLeoDecodeThreads) leo_decode16_staged_kernel(const __grid_constant__ LeoDecArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    const unsigned n = (unsigned)a.n, m = (unsigned)a.m;
    uint8_t *w = sm;
    uint8_t *tab = align_shared256(w + (size_t)n * kLeoTile);
    uint32_t *ctab = reinterpret_cast<uint32_t *>(tab + (size_t)kDecChunkSlots / 2 * 256);
    F16 fg;  // log-indexed tables for the per-row error-locator products
    fg.t = a.t16;
    fg.skew = a.skew;
    F16S fs;
    fs.t = a.t16;
    fs.skew = a.skew;
    fs.tab = (uint32_t)__cvta_generic_to_shared(tab);
    fs.ctab = (uint32_t)__cvta_generic_to_shared(ctab);
    fs.lo = 0;
    const long long off = (long long)blockIdx.x * kLeoTile;
    for (unsigned it = threadIdx.x; it < (n << F16::kQuadShift); it += blockDim.x) {
        const unsigned r = it >> F16::kQuadShift, c = it & (F16::kQuads - 1);
        int src = -1;
        if (r < (unsigned)a.p) src = a.k + (int)r;
        else if (r >= m && r < m + (unsigned)a.k) src = (int)(r - m);
        F16::Q v = F16::zero();
        if (src >= 0 && bit(a.present, src)) v = fg.mul(F16::ldg(a.shard[src] + off, c), a.errloc[r]);
        F16::st(w + (size_t)r * kLeoTile, c, v);
    }
    __syncthreads();
    ifft_staged(fs, w, tab, ctab, a.ts16, a.tw16, (unsigned)a.input_count, n);
    formal_derivative(w, n);
    fft_staged(fs, w, tab, ctab, a.ts16, a.tw16, m + (unsigned)a.k, n);
    const unsigned total = (unsigned)(a.k + a.p) << F16::kQuadShift;
    for (unsigned it = threadIdx.x; it < total; it += blockDim.x) {
        const int i = (int)(it >> F16::kQuadShift), c = (int)(it & (F16::kQuads - 1));
        if (!bit(a.write, i)) continue;
        const unsigned row = i >= a.k ? (unsigned)(i - a.k) : (unsigned)i + m;
        const uint32_t lm = F16::kMod - a.errloc[row];
        F16::stg(const_cast<uint8_t *>(a.shard[i]) + off, c, fg.mul(F16::ld(w + (size_t)row * kLeoTile, c), lm));
    }
}

// Shared bytes of the staged GF(2^16) encode (0 when it does not fit a CTA).
size_t staged_encode_smem(unsigned m) {
    const size_t bytes = EncLayout(m).bytes();
    return bytes <= 227u * 1024u ? bytes : 0;
}

// Formal derivative (leopard.go:620-623) on n rows in place.  Row x gains
// old[x + 2^b] for every b with bit b of x clear and ((x>>b)+1)<<b < n; all
// reads must see pre-derivative values, and they only reach higher rows, so
// rows are rewritten in ascending chunks with a barrier between the read
// and write phase of each chunk.
__device__ void formal_derivative(uint8_t *w, unsigned n) {
    constexpr unsigned kParts = kLeoTile / 16;  // 16-byte parts per row
    const unsigned rows_per_chunk = blockDim.x / kParts;
    const unsigned x_local = threadIdx.x / kParts, part = threadIdx.x % kParts;
    unsigned lg = 0;
    while ((2u << lg) <= n) lg++;  // n == 1 << lg
    for (unsigned base = 0; base < n; base += rows_per_chunk) {
        const unsigned x = base + x_local;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (x < n) {
            v = reinterpret_cast<const uint4 *>(w + (size_t)x * kLeoTile)[part];
            for (unsigned b = 0; b < lg; b++) {
                if (((x >> b) & 1u) || ((((x >> b) + 1) << b) >= n)) continue;
                const uint4 y = reinterpret_cast<const uint4 *>(w + (size_t)(x + (1u << b)) * kLeoTile)[part];
                v.x ^= y.x;
                v.y ^= y.y;
                v.z ^= y.z;
                v.w ^= y.w;
            }
        }
        __syncthreads();
        if (x < n) reinterpret_cast<uint4 *>(w + (size_t)x * kLeoTile)[part] = v;
        __syncthreads();
    }
}

// Decode (leopard.go:582-647 / leopard8.go:536-631).
template <class F>
__global__ void __launch_bounds__(kLeoDecodeThreads) leo_decode_kernel(const __grid_constant__ LeoDecArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    const bool gf8 = F::kQuads == 16;
    uint8_t *t8 = gf8 ? align_shared256(sm) : sm;
    uint8_t *w = gf8 ? t8 + kT8Bytes : sm;
    if (gf8) load_tables8<F>(t8, a.t8);
    __syncthreads();
    const F f = make_field<F>(a.t16, t8, a.skew);
    const long long off = (long long)blockIdx.x * kLeoTile;
    const unsigned n = (unsigned)a.n, m = (unsigned)a.m;
    // work <- received symbols scaled by their error locators; zeros elsewhere
    using Q = typename F::Q;
    for (unsigned it = threadIdx.x; it < (n << F::kQuadShift); it += blockDim.x) {
        const unsigned r = it >> F::kQuadShift, c = it & (F::kQuads - 1);
        int src = -1;
        if (r < (unsigned)a.p) src = a.k + (int)r;
        else if (r >= m && r < m + (unsigned)a.k) src = (int)(r - m);
        Q v = F::zero();
        if (src >= 0 && bit(a.present, src)) v = f.mul(F::ldg(a.shard[src] + off, c), a.errloc[r]);
        F::st(w + (size_t)r * kLeoTile, c, v);
    }
    __syncthreads();
    ifft_rows(f, w, (unsigned)a.input_count, n, -1);
    formal_derivative(w, n);
    fft_rows(f, w, m + (unsigned)a.k, n);
    // reveal: out = work * (modulus - errloc)
    const unsigned total = (unsigned)(a.k + a.p) << F::kQuadShift;
    for (unsigned it = threadIdx.x; it < total; it += blockDim.x) {
        const int i = (int)(it >> F::kQuadShift), c = (int)(it & (F::kQuads - 1));
        if (!bit(a.write, i)) continue;
        const unsigned row = i >= a.k ? (unsigned)(i - a.k) : (unsigned)i + m;
        const uint32_t lm = F::kMod - a.errloc[row];
        F::stg(const_cast<uint8_t *>(a.shard[i]) + off, c, f.mul(F::ld(w + (size_t)row * kLeoTile, c), lm));
    }
}

// ---- GF(2^16) geometries past one CTA's shared memory ---------------------
// Past 2048 shard pointers or 2048 transform rows (the reference allows up
// to 65536 shards, leopard.go:51-70) the transforms run over a work buffer
// in HBM, one row per pitch bytes in the reference's chunk layout, in
// passes.  A pass executes consecutive butterfly layers whose groups fit a
// set of at most kLeoSetRows rows: a set is rows base + t * d_lo, t < rows,
// where d_lo is the smallest distance of the pass (upper layers take sets of
// strided rows, lower layers sets of consecutive rows).  Each CTA loads one
// set's 64-byte column tile into shared memory, runs the pass's layers on it
// with multipliers indexed by global row numbers exactly as ifftDIT /
// fftDIT index them (leopard.go:650-736, :764-873), and writes it back.
constexpr int kLeoSetRows = 1024;  // 64 KB of shared memory per CTA
constexpr int kLeoPassThreads = 512;
constexpr int kLeoMaxLayers = 16;

struct LeoPassArgs {
    uint8_t *w;       // work rows
    long long pitch;  // bytes between work rows
    const uint16_t *skew, *t16;
    int n_layers;
    int d_lo;      // row stride inside a set
    int span;      // global rows one set's butterfly groups cover (set rows * d_lo)
    int set_rows;  // rows per set
    int sets;      // sets per CTA (they fill up to kLeoSetRows rows of shared memory)
    int mtrunc;    // butterfly groups starting at or above this row are skipped
    int skew_off;  // IFFT multiplier offset (-1 decoder, m-1+b*m encoder block b)
    int fft;       // 1: fftDIT layers, 0: ifftDIT layers
    int dist[kLeoMaxLayers];   // the layers' global distances, in execution order
    int radix[kLeoMaxLayers];  // 4 or 2
};

__global__ void __launch_bounds__(kLeoPassThreads) leo_pass16_kernel(const __grid_constant__ LeoPassArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    using Q = F16::Q;
    F16 f;
    f.t = a.t16;
    f.skew = a.skew;
    const long long col = (long long)blockIdx.x * kLeoTile;
    const unsigned d_lo = (unsigned)a.d_lo, rows = (unsigned)a.set_rows, nsets = (unsigned)a.sets;
    const unsigned set0 = blockIdx.y * nsets;
    // local row lr = s * rows + t is row t of set set0 + s: global row
    // g * span + o + t * d_lo with g, o the set's group and offset
    auto gstart = [&](unsigned s) { return (long long)((set0 + s) / d_lo) * a.span; };
    auto grow = [&](unsigned lr) {
        const unsigned s = lr / rows, t = lr % rows;
        return a.w + (gstart(s) + (set0 + s) % d_lo + (long long)t * d_lo) * a.pitch + col;
    };
    const unsigned all = nsets * rows;
    for (unsigned v = threadIdx.x; v < all * F16::kRowParts; v += blockDim.x)
        F16::row_in(sm + (size_t)(v / F16::kRowParts) * kLeoTile, grow(v / F16::kRowParts), v % F16::kRowParts);
    __syncthreads();
    for (int L = 0; L < a.n_layers; L++) {
        const unsigned dist = (unsigned)a.dist[L], ld = dist / d_lo;  // global and local distance
        const unsigned span_l = (unsigned)a.radix[L] * ld;           // local rows of one butterfly group
        const unsigned per_set = (rows / span_l) * ld;               // butterfly positions per set
        for (unsigned it = threadIdx.x; it < ((nsets * per_set) << F16::kQuadShift); it += blockDim.x) {
            const unsigned q = it >> F16::kQuadShift, c = it & (F16::kQuads - 1);
            const unsigned s = q / per_set, qs = q % per_set;
            const unsigned gl = qs / ld, i = s * rows + gl * span_l + qs % ld;
            const long long r = gstart(s) + (long long)gl * span_l * d_lo;  // group start, global
            if (a.radix[L] == 4) {
                if (r >= a.mtrunc) continue;
                uint8_t *p0 = sm + (size_t)i * kLeoTile;
                uint8_t *p1 = p0 + (size_t)ld * kLeoTile, *p2 = p1 + (size_t)ld * kLeoTile,
                        *p3 = p2 + (size_t)ld * kLeoTile;
                Q x0 = F16::ld(p0, c), x1 = F16::ld(p1, c), x2 = F16::ld(p2, c), x3 = F16::ld(p3, c);
                const long long iend = r + dist;
                if (a.fft) {
                    const uint32_t m01 = a.skew[iend - 1], m02 = a.skew[iend + dist - 1],
                                   m23 = a.skew[iend + 2 * dist - 1];
                    fft2(f, x0, x2, m02);
                    fft2(f, x1, x3, m02);
                    fft2(f, x0, x1, m01);
                    fft2(f, x2, x3, m23);
                } else {
                    const uint32_t m01 = a.skew[a.skew_off + iend], m02 = a.skew[a.skew_off + iend + dist],
                                   m23 = a.skew[a.skew_off + iend + 2 * dist];
                    ifft2(f, x0, x1, m01);
                    ifft2(f, x2, x3, m23);
                    ifft2(f, x0, x2, m02);
                    ifft2(f, x1, x3, m02);
                }
                F16::st(p0, c, x0);
                F16::st(p1, c, x1);
                F16::st(p2, c, x2);
                F16::st(p3, c, x3);
            } else {
                // radix 2: the IFFT's top layer (dist = n/2, every pair,
                // multiplier fftSkew[skew_off + dist]) or the FFT's last
                // (dist = 1, pairs (r, r+1) below mtrunc, multiplier fftSkew[r])
                if (a.fft && r >= a.mtrunc) continue;
                uint8_t *p0 = sm + (size_t)i * kLeoTile, *p1 = p0 + (size_t)ld * kLeoTile;
                Q x = F16::ld(p0, c), y = F16::ld(p1, c);
                if (a.fft) fft2(f, x, y, (uint32_t)a.skew[r]);
                else ifft2(f, x, y, (uint32_t)a.skew[a.skew_off + (long long)dist]);
                F16::st(p0, c, x);
                F16::st(p1, c, y);
            }
        }
        __syncthreads();
    }
    for (unsigned v = threadIdx.x; v < all * F16::kRowParts; v += blockDim.x)
        F16::row_out(grow(v / F16::kRowParts), sm + (size_t)(v / F16::kRowParts) * kLeoTile, v % F16::kRowParts);
}

// Formal derivative (leopard.go:620-623) on rows [c0, c0 + crows) of the
// work buffer: row x gains old[x + 2^b] for every b with bit b of x clear and
// ((x>>b)+1)<<b < n.  Launched for ascending chunks: rows past the chunk are
// still old, and inside it every read comes before the barrier that precedes
// the writes.  XOR is bytewise, so the raw layout is used as it is.
__global__ void __launch_bounds__(kLeoPassThreads) leo_deriv16_chunk_kernel(uint8_t *w, long long pitch, unsigned n,
                                                                           unsigned c0, unsigned crows) {
    extern __shared__ __align__(16) uint8_t sm[];  // crows * 64 bytes of new values
    const long long col = (long long)blockIdx.x * kLeoTile;
    unsigned lg = 0;
    while ((2u << lg) <= n) lg++;
    for (unsigned v = threadIdx.x; v < crows * 4; v += blockDim.x) {
        const unsigned x = c0 + v / 4, part = v % 4;
        uint4 acc = reinterpret_cast<const uint4 *>(w + (long long)x * pitch + col)[part];
        for (unsigned b = 0; b < lg; b++) {
            if (((x >> b) & 1u) || ((((x >> b) + 1) << b) >= n)) continue;
            const uint4 y = reinterpret_cast<const uint4 *>(w + (long long)(x + (1u << b)) * pitch + col)[part];
            acc.x ^= y.x;
            acc.y ^= y.y;
            acc.z ^= y.z;
            acc.w ^= y.w;
        }
        reinterpret_cast<uint4 *>(sm)[v] = acc;
    }
    __syncthreads();
    for (unsigned v = threadIdx.x; v < crows * 4; v += blockDim.x)
        reinterpret_cast<uint4 *>(w + (long long)(c0 + v / 4) * pitch + col)[v % 4] = reinterpret_cast<uint4 *>(sm)[v];
}

// Work rows [0, rows) <- shards [first, first + cnt) (raw copy), zero past cnt.
__global__ void leo_rows_in_kernel(uint8_t *w, long long pitch, const uint8_t *const *shard, int first, int cnt,
                                   int rows, long long vecs_per_row) {
    const long long total = (long long)rows * vecs_per_row;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(v / vecs_per_row);
        const long long e = v % vecs_per_row;
        const uint4 x = r < cnt ? __ldcs(reinterpret_cast<const uint4 *>(shard[first + r]) + e) : make_uint4(0, 0, 0, 0);
        reinterpret_cast<uint4 *>(w + (long long)r * pitch)[e] = x;
    }
}

// Shards [first, first + cnt) <- work rows [0, cnt).
__global__ void leo_rows_out_kernel(const uint8_t *w, long long pitch, const uint8_t *const *shard, int first,
                                    int cnt, long long vecs_per_row) {
    const long long total = (long long)cnt * vecs_per_row;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(v / vecs_per_row);
        const long long e = v % vecs_per_row;
        __stcs(reinterpret_cast<uint4 *>(const_cast<uint8_t *>(shard[first + r])) + e,
               reinterpret_cast<const uint4 *>(w + (long long)r * pitch)[e]);
    }
}

// Decoder input (leopard.go:586-605): work row r = received shard times its
// error locator (parity at rows [0, p), data at [m, m+k)), zero elsewhere.
__global__ void leo_dec_load16_kernel(uint8_t *w, long long pitch, const uint8_t *const *shard,
                                      const uint32_t *present, const uint16_t *errloc, const uint16_t *t16,
                                      const uint16_t *skew, int k, int p, int m, int n, long long quads_per_row) {
    F16 f;
    f.t = t16;
    f.skew = skew;
    const long long total = (long long)n * quads_per_row;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(v / quads_per_row);
        const long long qq = v % quads_per_row, chunk = qq / F16::kQuads;
        const int c = (int)(qq % F16::kQuads);
        int src = -1;
        if (r < p) src = k + r;
        else if (r >= m && r < m + k) src = r - m;
        F16::Q x = F16::zero();
        if (src >= 0 && bit(present, src)) x = f.mul(F16::ldg(shard[src] + chunk * kLeoTile, c), errloc[r]);
        F16::stg(w + (long long)r * pitch + chunk * kLeoTile, c, x);
    }
}

// Reveal (leopard.go:636-647): shard i <- work row times (modulus - errloc).
__global__ void leo_reveal16_kernel(const uint8_t *w, long long pitch, const uint8_t *const *shard,
                                    const uint32_t *write, const uint16_t *errloc, const uint16_t *t16,
                                    const uint16_t *skew, int k, int total, int m, long long quads_per_row) {
    F16 f;
    f.t = t16;
    f.skew = skew;
    const long long all = (long long)total * quads_per_row;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < all;
         v += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(v / quads_per_row);
        if (!bit(write, i)) continue;
        const long long qq = v % quads_per_row, chunk = qq / F16::kQuads;
        const int c = (int)(qq % F16::kQuads);
        const unsigned row = i >= k ? (unsigned)(i - k) : (unsigned)i + (unsigned)m;
        const uint32_t lm = F16::kMod - errloc[row];
        F16::stg(const_cast<uint8_t *>(shard[i]) + chunk * kLeoTile, c,
                 f.mul(F16::ldg(w + (long long)row * pitch + chunk * kLeoTile, c), lm));
    }
}

// Error locators of an erasure pattern (leopard.go:468-510,
// leopard8.go:465-513).  The reference puts ones at erased rows (parity rows
// first, the padding rows p..m-1, data rows at offset m), takes a 2^BITS-point
// Walsh-Hadamard transform, multiplies by FWHT(log) mod (2^BITS - 1) and
// transforms again, and the decoder reads only the first n = ceilPow2(m+k)
// results.  The ones all sit below n, so the first transform is n-periodic,
// and summing the second transform's input over the high bits leaves an
// n-point transform: errloc[0..n) = WHT_n(WHT_n(ones) * W_n) with
// W_n[i] = sum_h FWHT(log)[h*n + i] mod (2^BITS - 1) (built once per field).
// The results are congruent to the reference's modulo 2^BITS - 1, which is
// all the log-domain products that consume them depend on.
template <int BITS>
__device__ __forceinline__ uint32_t wh_add(uint32_t a, uint32_t b) {
    const uint32_t s = a + b;  // partial reduction, may give the modulus (leopard.go:1001-1006)
    return (s + (s >> BITS)) & ((1u << BITS) - 1);
}
template <int BITS>
__device__ __forceinline__ uint32_t wh_sub(uint32_t a, uint32_t b) {
    const unsigned long long d = (unsigned long long)a - (unsigned long long)b;  // wraps like Go's uint
    return (uint32_t)((d + (d >> BITS)) & ((1u << BITS) - 1));
}

// n-point Walsh-Hadamard transform in shared memory (n a power of two).
template <int BITS>
__device__ void wht_shared(uint16_t *v, unsigned n) {
    unsigned dist = 1, dist4 = 4, ld = 0;
    for (; dist4 <= n; dist = dist4, dist4 <<= 2, ld += 2) {
        for (unsigned it = threadIdx.x; it < (n >> 2); it += blockDim.x) {
            const unsigned i = ((it >> ld) << (ld + 2)) + (it & (dist - 1));
            const uint32_t t0 = v[i], t1 = v[i + dist], t2 = v[i + 2 * dist], t3 = v[i + 3 * dist];
            const uint32_t a = wh_add<BITS>(t0, t1), b = wh_sub<BITS>(t0, t1);
            const uint32_t c = wh_add<BITS>(t2, t3), d = wh_sub<BITS>(t2, t3);
            v[i] = (uint16_t)wh_add<BITS>(a, c);
            v[i + 2 * dist] = (uint16_t)wh_sub<BITS>(a, c);
            v[i + dist] = (uint16_t)wh_add<BITS>(b, d);
            v[i + 3 * dist] = (uint16_t)wh_sub<BITS>(b, d);
        }
        __syncthreads();
    }
    if (dist < n) {  // odd log2(n): one radix-2 layer with dist == n / 2
        for (unsigned i = threadIdx.x; i < dist; i += blockDim.x) {
            const uint32_t t0 = v[i], t1 = v[i + dist];
            v[i] = (uint16_t)wh_add<BITS>(t0, t1);
            v[i + dist] = (uint16_t)wh_sub<BITS>(t0, t1);
        }
        __syncthreads();
    }
}

constexpr int kLeoMaxAllShards = 65536;  // leopard.go:51-70

struct LeoErrArgs {
    uint32_t present[kLeoMaxAllShards / 32];
    int k, p, m, n;
    const uint16_t *fold;  // W_n
    uint16_t *out;
};

constexpr int kErrLocThreads = 512;

template <int BITS>
__global__ void __launch_bounds__(kErrLocThreads) leo_errloc_kernel(const __grid_constant__ LeoErrArgs a) {
    constexpr uint32_t kMod = (1u << BITS) - 1;
    extern __shared__ __align__(16) uint16_t el[];  // n entries (at most 65536: 128 KB)
    const unsigned m = (unsigned)a.m, k = (unsigned)a.k, p = (unsigned)a.p, n = (unsigned)a.n;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        uint16_t v = 0;
        if (i < p) v = bit(a.present, (int)(k + i)) ? 0 : 1;
        else if (i < m) v = 1;
        else if (i < m + k) v = bit(a.present, (int)(i - m)) ? 0 : 1;
        el[i] = v;
    }
    __syncthreads();
    wht_shared<BITS>(el, n);
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) el[i] = (uint16_t)(((uint32_t)el[i] * a.fold[i]) % kMod);
    __syncthreads();
    wht_shared<BITS>(el, n);
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) a.out[i] = el[i];
}

// W_b for b = 0..max_bits, W_b stored at [2^b, 2^(b+1)).
template <int BITS>
std::vector<uint16_t> fold_walsh(const std::vector<uint16_t> &walsh, int max_bits) {
    const unsigned order = 1u << BITS, mod = order - 1;
    std::vector<uint16_t> out(2u << max_bits, 0);
    for (int b = 0; b <= max_bits; b++) {
        const unsigned n = 1u << b;
        for (unsigned i = 0; i < n; i++) {
            unsigned long long acc = 0;
            for (unsigned h = 0; h < order / n; h++) acc += walsh[h * n + i];
            out[n + i] = (uint16_t)(acc % mod);
        }
    }
    return out;
}

// Builds the [65536][kT16Stride] split product tables of F16:
// mulLog(j, lm), mulLog(j << 6, lm), mulLog(j << 12, lm) (leopard.go:1008-1014).
__global__ void build_t16(uint16_t *t, const uint16_t *log, const uint16_t *exp) {
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 65536u * kT16Stride;
         idx += gridDim.x * blockDim.x) {
        const unsigned lm = idx / kT16Stride, j = idx % kT16Stride;
        unsigned x = 0;
        if (j < 64) x = j;
        else if (j < 128) x = (j - 64) << 6;
        else if (j < 144) x = (j - 128) << 12;
        uint16_t v = 0;
        if (x) {
            unsigned s = (unsigned)log[x] + lm;
            s = (s + (s >> 16)) & 0xFFFF;  // addMod partial reduction (leopard.go:1001-1006)
            v = exp[s];
        }
        t[idx] = v;
    }
}

// Builds the skew-ordered nibble tables of F16S: entry [i][q][e] =
// mulLog(e << 4q, fftSkew[i]), zero when fftSkew[i] is the modulus.
__global__ void build_ts16(uint16_t *t, const uint16_t *skew, const uint16_t *log, const uint16_t *exp) {
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 65535u * 64u; idx += gridDim.x * blockDim.x) {
        const unsigned i = idx >> 6, q = (idx >> 4) & 3, e = idx & 15;
        const unsigned lm = skew[i], x = e << (4 * q);
        uint16_t v = 0;
        if (x && lm != 65535u) {
            unsigned s = (unsigned)log[x] + lm;
            s = (s + (s >> 16)) & 0xFFFF;
            v = exp[s];
        }
        t[idx] = v;
    }
}

// Builds the wide tables of F16W: row j serves fftSkew index 4j + 3 (zero
// past the table or where the skew is the modulus); entries mulLog(e, lm)
// (e < 64), mulLog(e << 6, lm) and mulLog(e << 11, lm) (e < 32).
__global__ void build_tw16(uint16_t *t, const uint16_t *skew, const uint16_t *log, const uint16_t *exp) {
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < 16384u * 128u; idx += gridDim.x * blockDim.x) {
        const unsigned j = idx >> 7, e = idx & 127, i = 4 * j + 3;
        const unsigned lm = i < 65535u ? skew[i] : 65535u;
        const unsigned x = e < 64 ? e : (e < 96 ? (e - 64) << 6 : (e - 96) << 11);
        uint16_t v = 0;
        if (x && lm != 65535u) {
            unsigned s = (unsigned)log[x] + lm;
            s = (s + (s >> 16)) & 0xFFFF;
            v = exp[s];
        }
        t[idx] = v;
    }
}

int ensure_tables(rsgpu_encoder *enc) {
    rsgpu_ctx *ctx = enc->ctx;
    if (enc->leo && enc->leo->device == ctx->device) return RS_OK;
    if (ctx->leo) {
        enc->leo = ctx->leo;
        return RS_OK;
    }
    auto st = std::make_shared<LeoState>();
    st->device = ctx->device;
    const Leo16 &f16 = Leo16::get();
    const Leo8 &f8 = Leo8::get();
    RS_CUDA(cudaMalloc(&st->skew16, 65535 * 2));
    RS_CUDA(cudaMalloc(&st->t16, 65536ull * kT16Stride * 2));
    RS_CUDA(cudaMalloc(&st->skew8, 255 * 2));
    RS_CUDA(cudaMalloc(&st->t8, kT8Bytes));
    RS_CUDA(cudaMemcpy(st->skew16, f16.skew.data(), 65535 * 2, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemcpy(st->skew8, f8.skew.data(), 255 * 2, cudaMemcpyHostToDevice));
    {
        const std::vector<uint16_t> w16 = fold_walsh<16>(f16.walsh, 16), w8 = fold_walsh<8>(f8.walsh, 8);
        RS_CUDA(cudaMalloc(&st->fold16, w16.size() * 2));
        RS_CUDA(cudaMalloc(&st->fold8, w8.size() * 2));
        RS_CUDA(cudaMemcpy(st->fold16, w16.data(), w16.size() * 2, cudaMemcpyHostToDevice));
        RS_CUDA(cudaMemcpy(st->fold8, w8.data(), w8.size() * 2, cudaMemcpyHostToDevice));
    }
    std::vector<uint8_t> t8(kT8Bytes);
    for (unsigned lm = 0; lm < 256; lm++)
        for (unsigned q = 0; q < 2; q++)
            for (unsigned e = 0; e < 16; e++) t8[lm * 32 + q * 16 + e] = (uint8_t)f8.mul_log((uint16_t)(e << (4 * q)), (uint16_t)lm);
    RS_CUDA(cudaMemcpy(st->t8, t8.data(), kT8Bytes, cudaMemcpyHostToDevice));
    uint16_t *dlog = nullptr, *dexp = nullptr;
    RS_CUDA(cudaMalloc(&dlog, 65536 * 2));
    RS_CUDA(cudaMalloc(&dexp, 65536 * 2));
    RS_CUDA(cudaMemcpy(dlog, f16.log.data(), 65536 * 2, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemcpy(dexp, f16.exp.data(), 65536 * 2, cudaMemcpyHostToDevice));
    build_t16<<<1024, 256, 0, ctx->stream>>>(st->t16, dlog, dexp);
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaMalloc(&st->ts16, 65535ull * 64 * 2));
    build_ts16<<<1024, 256, 0, ctx->stream>>>(st->ts16, st->skew16, dlog, dexp);
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaMalloc(&st->tw16, 16384ull * 128 * 2));
    build_tw16<<<1024, 256, 0, ctx->stream>>>(st->tw16, st->skew16, dlog, dexp);
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaFree(dlog);
    cudaFree(dexp);
    ctx->leo = st;
    enc->leo = st;
    return RS_OK;
}

bool is16(const rsgpu_encoder *enc) { return enc->codec == RS_CODEC_LEOPARD16; }

// Largest skew index the encoder reads must stay inside fftSkew (the
// reference indexes past it otherwise, leopard8.go:151,201-233).
bool encode_fits(const rsgpu_encoder *enc) {
    const unsigned m = ceil_pow2((unsigned)enc->p);
    const unsigned blocks = ((unsigned)enc->k + m - 1) / m;
    const unsigned max_index = (m - 1) + (blocks - 1) * m + (m - 1);
    return max_index < (is16(enc) ? 65535u : 255u);
}

// The kernels move shard data in 16-byte (encode) and 4-byte (decode)
// vectors, so every buffer they touch must be 16-byte aligned.
bool shards_aligned(const uint8_t *const *shards, int n) {
    for (int i = 0; i < n; i++)
        if (shards[i] && (reinterpret_cast<uintptr_t>(shards[i]) & 15u)) return false;
    return true;
}

template <class K>
int set_smem(K kern, size_t bytes) {
    RS_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return RS_OK;
}

// ---- GF(2^16) past one CTA: passes over a work buffer in HBM --------------

// The layers of an n-row ifftDIT (ascending radix-4 distances, then one
// radix-2 layer at n/2 when log2 n is odd) or fftDIT (descending radix-4
// distances, then one radix-2 layer at distance 1), exactly as
// ifft_rows / fft_rows run them, grouped into passes whose sets stay within
// kLeoSetRows rows.
std::vector<LeoPassArgs> plan_passes(unsigned n, bool fft) {
    std::vector<std::pair<unsigned, int>> layers;  // (distance, radix)
    if (!fft) {
        unsigned dist = 1, dist4 = 4;
        for (; dist4 <= n; dist = dist4, dist4 <<= 2) layers.push_back({dist, 4});
        if (dist < n) layers.push_back({dist, 2});
    } else {
        unsigned dist4 = n, dist = n >> 2;
        for (; dist != 0; dist4 = dist, dist >>= 2) layers.push_back({dist, 4});
        if (dist4 == 2) layers.push_back({1u, 2});
    }
    std::vector<LeoPassArgs> passes;
    for (size_t first = 0; first < layers.size();) {
        unsigned lo = layers[first].first, span = layers[first].first * layers[first].second;
        size_t end = first + 1;
        while (end < layers.size() && end - first < (size_t)kLeoMaxLayers) {
            const unsigned nlo = std::min(lo, layers[end].first);
            const unsigned nspan = std::max(span, layers[end].first * (unsigned)layers[end].second);
            if (nspan / nlo > (unsigned)kLeoSetRows) break;
            lo = nlo;
            span = nspan;
            end++;
        }
        LeoPassArgs a;
        memset(&a, 0, sizeof a);
        a.n_layers = (int)(end - first);
        a.d_lo = (int)lo;
        a.span = (int)span;
        a.set_rows = (int)(span / lo);
        a.fft = fft ? 1 : 0;
        for (size_t L = first; L < end; L++) {
            a.dist[L - first] = (int)layers[L].first;
            a.radix[L - first] = layers[L].second;
        }
        passes.push_back(a);
        first = end;
    }
    return passes;
}

// Runs an n-row transform on work rows w (pitch bytes apart, `size` bytes
// of every row processed).
int run_passes(const LeoState &L, uint8_t *w, long long pitch, size_t size, unsigned n, bool fft, int mtrunc,
               int skew_off, cudaStream_t st) {
    int rc = set_smem(leo_pass16_kernel, (size_t)kLeoSetRows * kLeoTile);  // per device, so on every call
    if (rc) return rc;
    for (LeoPassArgs a : plan_passes(n, fft)) {
        a.w = w;
        a.pitch = pitch;
        a.skew = L.skew16;
        a.t16 = L.t16;
        a.mtrunc = mtrunc;
        a.skew_off = skew_off;
        const unsigned nsets = n / (unsigned)a.set_rows;
        a.sets = (int)std::min(nsets, (unsigned)kLeoSetRows / (unsigned)a.set_rows);
        const dim3 grid((unsigned)(size / kLeoTile), nsets / (unsigned)a.sets);
        leo_pass16_kernel<<<grid, kLeoPassThreads, (size_t)a.sets * a.set_rows * kLeoTile, st>>>(a);
        RS_CUDA(cudaGetLastError());
    }
    return RS_OK;
}

// Grid of the row-copy / row-map kernels.
int rows_grid(long long items) { return (int)std::max(1LL, std::min((items + 255) / 256, 148LL * 16)); }

// Stream-ordered scratch from the context pool, freed behind the call's work.
struct PoolScratch {
    cudaStream_t st;
    cudaMemPool_t pool;
    std::vector<void *> blocks;
    int get(void **p, size_t bytes) {
        RS_CUDA(cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st));
        blocks.push_back(*p);
        return RS_OK;
    }
    ~PoolScratch() {
        for (void *b : blocks) cudaFreeAsync(b, st);
    }
};

// Encode (leopard.go:169-270) for GF(2^16) geometries past one CTA: work rows
// [0, m) accumulate, [m, 2m) hold each later data block; every block's IFFT
// and the final FFT run as passes.
int leo_encode_large(rsgpu_encoder *enc, uint8_t *const *shards, size_t size, cudaStream_t st) {
    const int k = enc->k, p = enc->p, total = enc->total;
    const unsigned m = ceil_pow2((unsigned)p);
    const LeoState &L = *enc->leo;
    PoolScratch sc{st, enc->ctx->pool, {}};
    const uint8_t **dptr = nullptr;
    uint8_t *w = nullptr;
    int rc = sc.get((void **)&dptr, sizeof(void *) * (size_t)total);
    if (!rc) rc = sc.get((void **)&w, (size_t)2 * m * size);
    if (rc) return rc;
    RS_CUDA(cudaMemcpyAsync(dptr, shards, sizeof(void *) * (size_t)total, cudaMemcpyHostToDevice, st));
    const long long pitch = (long long)size, vecs = (long long)(size / 16);
    uint8_t *acc = w, *tmp = w + (size_t)m * size;
    for (int b = 0; b * (int)m < k; b++) {
        const int start = b * (int)m, cnt = std::min((int)m, k - start);
        uint8_t *dst = b == 0 ? acc : tmp;
        leo_rows_in_kernel<<<rows_grid((long long)m * vecs), 256, 0, st>>>(dst, pitch, dptr, start, cnt, (int)m, vecs);
        RS_CUDA(cudaGetLastError());
        rc = run_passes(L, dst, pitch, size, m, false, cnt, (int)m - 1 + b * (int)m, st);
        if (rc) return rc;
        if (b > 0) RS_CUDA(launch_xor(st, enc->ctx->info, tmp, acc, (size_t)m * size));
    }
    rc = run_passes(L, acc, pitch, size, m, true, p, 0, st);
    if (rc) return rc;
    leo_rows_out_kernel<<<rows_grid((long long)p * vecs), 256, 0, st>>>(acc, pitch, dptr, k, p, vecs);
    RS_CUDA(cudaGetLastError());
    return RS_OK;
}

// Decode (leopard.go:582-647) for GF(2^16) geometries past one CTA, given the
// first n error locators on the device.
int leo_decode_large(rsgpu_encoder *enc, uint8_t *const *shards, const std::vector<uint32_t> &present,
                     const std::vector<uint32_t> &write, const uint16_t *d_el, unsigned m, unsigned n,
                     int input_count, size_t size, cudaStream_t st) {
    const int k = enc->k, p = enc->p, total = enc->total;
    const LeoState &L = *enc->leo;
    PoolScratch sc{st, enc->ctx->pool, {}};
    const uint8_t **dptr = nullptr;
    uint32_t *dpres = nullptr, *dwrite = nullptr;
    uint8_t *w = nullptr;
    int rc = sc.get((void **)&dptr, sizeof(void *) * (size_t)total);
    if (!rc) rc = sc.get((void **)&dpres, present.size() * 4);
    if (!rc) rc = sc.get((void **)&dwrite, write.size() * 4);
    if (!rc) rc = sc.get((void **)&w, (size_t)n * size);
    if (rc) return rc;
    RS_CUDA(cudaMemcpyAsync(dptr, shards, sizeof(void *) * (size_t)total, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dpres, present.data(), present.size() * 4, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dwrite, write.data(), write.size() * 4, cudaMemcpyHostToDevice, st));
    const long long pitch = (long long)size, quads = (long long)(size / kLeoTile) * F16::kQuads;
    leo_dec_load16_kernel<<<rows_grid((long long)n * quads), 256, 0, st>>>(w, pitch, dptr, dpres, d_el, L.t16,
                                                                           L.skew16, k, p, (int)m, (int)n, quads);
    RS_CUDA(cudaGetLastError());
    rc = run_passes(L, w, pitch, size, n, false, input_count, -1, st);
    if (rc) return rc;
    const unsigned crows = std::min(n, (unsigned)kLeoSetRows);
    rc = set_smem(leo_deriv16_chunk_kernel, (size_t)kLeoSetRows * kLeoTile);
    if (rc) return rc;
    for (unsigned c0 = 0; c0 < n; c0 += crows) {
        leo_deriv16_chunk_kernel<<<(unsigned)(size / kLeoTile), kLeoPassThreads, (size_t)crows * kLeoTile, st>>>(
            w, pitch, n, c0, crows);
        RS_CUDA(cudaGetLastError());
    }
    rc = run_passes(L, w, pitch, size, n, true, (int)m + k, 0, st);
    if (rc) return rc;
    leo_reveal16_kernel<<<rows_grid((long long)total * quads), 256, 0, st>>>(w, pitch, dptr, dwrite, d_el, L.t16,
                                                                             L.skew16, k, total, (int)m, quads);
    RS_CUDA(cudaGetLastError());
    return RS_OK;
}

}  // namespace

int leo_create(rsgpu_encoder *enc) {
    if (enc->k <= 0 || enc->p <= 0) return RS_ERR_INV_SHARD_NUM;
    if (enc->k + enc->p > 65536) return RS_ERR_MAX_SHARD_NUM;
    if (!is16(enc) && ceil_pow2((unsigned)enc->p) + (unsigned)enc->k > 256) return RS_ERR_MAX_SHARD_NUM;
    if (!encode_fits(enc)) return RS_ERR_MAX_SHARD_NUM;
    return RS_OK;
}

int leo_encode_enqueue(rsgpu_encoder *enc, uint8_t *const *shards, size_t size, cudaStream_t st) {
    if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
    const unsigned m = ceil_pow2((unsigned)enc->p);
    if (!shards_aligned(shards, enc->total)) {
        set_error("leopard encode: shard buffers must be 16-byte aligned");
        return RS_ERR_NOT_SUPPORTED;
    }
    const bool fits_cta = enc->total <= kLeoMaxShards && 2 * m <= kLeoMaxRows;
    if (!fits_cta && !is16(enc)) {  // not reachable by a valid GF(2^8) geometry (k+p <= 256)
        set_error("leopard encode: geometry exceeds the shared-memory transform");
        return RS_ERR_NOT_SUPPORTED;
    }
    int rc = ensure_tables(enc);
    if (rc) return rc;
    if (!fits_cta) return leo_encode_large(enc, shards, size, st ? st : enc->ctx->stream);
    LeoEncArgs a;
    memset(&a, 0, sizeof a);
    for (int i = 0; i < enc->total; i++) a.shard[i] = shards[i];
    a.k = enc->k;
    a.p = enc->p;
    a.m = (int)m;
    a.size = (long long)size;
    const bool g16 = is16(enc);
    a.skew = g16 ? enc->leo->skew16 : enc->leo->skew8;
    a.t16 = enc->leo->t16;
    a.ts16 = enc->leo->ts16;
    a.tw16 = enc->leo->tw16;
    a.t8 = enc->leo->t8;
    const size_t smem = (size_t)2 * m * kLeoTile + (g16 ? 0 : kT8Bytes + kT8Slack);
    const int grid = (int)(size / kLeoTile);
    if (!st) st = enc->ctx->stream;
    const size_t staged = g16 ? staged_encode_smem(m) : 0;
    if (staged && m >= 4) {
        rc = set_smem(leo_encode16_staged_kernel, staged);
        if (rc) return rc;
        const int threads = (int)std::min<unsigned>(kLeoEncThreadsMax, std::max(64u, 2 * m));
        leo_encode16_staged_kernel<<<grid, threads, staged, st>>>(a);
    } else if (g16) {
        rc = set_smem(leo_encode_kernel<F16>, smem);
        if (rc) return rc;
        leo_encode_kernel<F16><<<grid, kLeoThreads, smem, st>>>(a);
    } else {
        rc = set_smem(leo_encode_kernel<F8>, smem);
        if (rc) return rc;
        leo_encode_kernel<F8><<<grid, kLeoThreads, smem, st>>>(a);
    }
    RS_CUDA(cudaGetLastError());
    return RS_OK;
}

int leo_encode(rsgpu_encoder *enc, uint8_t *const *shards, size_t size) {
    int rc = leo_encode_enqueue(enc, shards, size);
    if (rc) return rc;
    RS_CUDA(cudaStreamSynchronize(enc->ctx->stream));
    return RS_OK;
}

// Checks of leopard.go:421-460 shared by the device and host entry points.
static int decode_checks(rsgpu_encoder *enc, const uint8_t *present, size_t size, int recover_all,
                         bool *nothing) {
    int np = 0, dp = 0;
    for (int i = 0; i < enc->total; i++)
        if (present[i]) {
            np++;
            if (i < enc->k) dp++;
        }
    *nothing = false;
    if (np == 0 || size == 0) return RS_ERR_SHARD_NO_DATA;
    if (np == enc->total || (!recover_all && dp == enc->k)) {
        *nothing = true;
        return RS_OK;
    }
    if (np < enc->k) return RS_ERR_TOO_FEW_SHARDS;
    if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
    return RS_OK;
}

int leo_reconstruct_enqueue(rsgpu_encoder *enc, uint8_t *const *shards, const uint8_t *present,
                            size_t size, int recover_all, cudaStream_t st) {
    bool nothing = false;
    int rc = decode_checks(enc, present, size, recover_all, &nothing);
    if (rc || nothing) return rc;
    const int k = enc->k, p = enc->p, total = enc->total;
    const unsigned m = ceil_pow2((unsigned)p), n = ceil_pow2(m + (unsigned)k);
    const bool g16 = is16(enc);
    const bool fits_cta = total <= kLeoMaxShards && n <= (unsigned)kLeoMaxRows;
    if (!fits_cta && !g16) {  // not reachable by a valid GF(2^8) geometry (k+p <= 256)
        set_error("leopard decode: geometry exceeds the shared-memory transform");
        return RS_ERR_NOT_SUPPORTED;
    }
    if (!shards_aligned(shards, total)) {
        set_error("leopard reconstruct: shard buffers must be 16-byte aligned");
        return RS_ERR_NOT_SUPPORTED;
    }
    rc = ensure_tables(enc);
    if (rc) return rc;
    int input_count = p;
    for (int i = 0; i < k; i++)
        if (present[i]) input_count = (int)m + i + 1;
    const int end = recover_all ? total : k;
    std::vector<uint32_t> pres((total + 31) / 32, 0), write((total + 31) / 32, 0);
    for (int i = 0; i < total; i++) {
        if (present[i]) pres[i >> 5] |= 1u << (i & 31);
        else if (i < end) {
            if (!shards[i]) return RS_ERR_INVALID_INPUT;
            write[i >> 5] |= 1u << (i & 31);
        }
    }
    if (!st) st = enc->ctx->stream;
    // error locators: from the per-pattern cache, else computed on the device
    // into stream-ordered scratch (kept in the cache while it has room, else
    // freed behind the decode)
    if (!enc->errlocs) {
        enc->errlocs = std::make_shared<LeoErrLocCache>();
        enc->errlocs->device = enc->ctx->device;
    }
    LeoErrLocCache &cache = *enc->errlocs;
    uint16_t *d_el = nullptr;
    {
        std::lock_guard<std::mutex> lk(cache.mu);
        auto it = cache.map.find(pres);
        if (it != cache.map.end()) {
            d_el = it->second.d;
            RS_CUDA(cudaStreamWaitEvent(st, it->second.ready, 0));
        }
    }
    bool owned = false;  // true: scratch to free after the decode
    if (!d_el) {
        RS_CUDA(cudaMallocFromPoolAsync((void **)&d_el, (size_t)n * sizeof(uint16_t), enc->ctx->pool, st));
        owned = true;
        auto ea = std::unique_ptr<LeoErrArgs>(new LeoErrArgs());
        memset(ea.get(), 0, sizeof *ea);
        memcpy(ea->present, pres.data(), pres.size() * 4);
        ea->k = k;
        ea->p = p;
        ea->m = (int)m;
        ea->n = (int)n;
        ea->out = d_el;
        ea->fold = (g16 ? enc->leo->fold16 : enc->leo->fold8) + n;
        const size_t el_smem = (size_t)n * sizeof(uint16_t);
        if (g16) rc = set_smem(leo_errloc_kernel<16>, el_smem > (48u << 10) ? el_smem : (48u << 10));
        if (rc) {
            cudaFreeAsync(d_el, st);
            return rc;
        }
        if (g16) leo_errloc_kernel<16><<<1, kErrLocThreads, el_smem, st>>>(*ea);
        else leo_errloc_kernel<8><<<1, kErrLocThreads, el_smem, st>>>(*ea);
        rc = cuda_status(cudaGetLastError(), "leo_errloc_kernel");
        if (rc) {
            cudaFreeAsync(d_el, st);
            return rc;
        }
        std::lock_guard<std::mutex> lk(cache.mu);
        if (cache.map.size() < kErrLocCacheCap && !cache.map.count(pres)) {
            cudaEvent_t ev = nullptr;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
                if (cudaEventRecord(ev, st) == cudaSuccess) {
                    cache.map[pres] = LeoErrLocCache::Entry{d_el, ev};
                    owned = false;
                } else {
                    cudaEventDestroy(ev);
                }
            }
        }
    }
    if (!fits_cta) {
        rc = leo_decode_large(enc, shards, pres, write, d_el, m, n, input_count, size, st);
        if (owned) cudaFreeAsync(d_el, st);
        return rc;
    }
    static_assert(sizeof(LeoDecArgs) < 32000, "kernel parameter limit");
    auto a = std::unique_ptr<LeoDecArgs>(new LeoDecArgs());
    memset(a.get(), 0, sizeof *a);
    for (int i = 0; i < total; i++) a->shard[i] = shards[i];
    memcpy(a->present, pres.data(), pres.size() * 4);
    memcpy(a->write, write.data(), write.size() * 4);
    a->errloc = d_el;
    a->k = k;
    a->p = p;
    a->m = (int)m;
    a->n = (int)n;
    a->input_count = input_count;
    a->size = (long long)size;
    a->skew = g16 ? enc->leo->skew16 : enc->leo->skew8;
    a->t16 = enc->leo->t16;
    a->ts16 = enc->leo->ts16;
    a->tw16 = enc->leo->tw16;
    a->t8 = enc->leo->t8;
    const size_t smem = g16 ? (size_t)n * kLeoTile + kDecTableBytes + 256 : (size_t)n * kLeoTile + kT8Bytes + kT8Slack;
    const int grid = (int)(size / kLeoTile);
    rc = g16 ? set_smem(leo_decode16_staged_kernel, smem) : set_smem(leo_decode_kernel<F8>, smem);
    if (rc == RS_OK) {
        if (g16) leo_decode16_staged_kernel<<<grid, kLeoDecodeThreads, smem, st>>>(*a);
        else leo_decode_kernel<F8><<<grid, kLeoDecodeThreads, smem, st>>>(*a);
        rc = cuda_status(cudaGetLastError(), "leo_decode_kernel");
    }
    if (owned) cudaFreeAsync(d_el, st);
    return rc;
}

int leo_reconstruct(rsgpu_encoder *enc, uint8_t **shards, const uint8_t *present, size_t size,
                    int recover_all, uint8_t *written) {
    if (written) memset(written, 0, (size_t)enc->total);
    bool nothing = false;
    int rc = decode_checks(enc, present, size, recover_all, &nothing);
    if (rc || nothing) return rc;
    const int end = recover_all ? enc->total : enc->k;
    if (!shards_aligned(shards, enc->total)) {  // before allocating anything
        set_error("leopard reconstruct: shard buffers must be 16-byte aligned");
        return RS_ERR_NOT_SUPPORTED;
    }
    for (int i = 0; i < enc->total; i++) {
        if (present[i]) {
            if (!shards[i]) return RS_ERR_SHARD_SIZE;
        } else if (i < end && !shards[i]) {  // allocate like leopard.go:528-534
            void *pnew = nullptr;
            RS_CUDA(cudaMalloc(&pnew, size));
            shards[i] = (uint8_t *)pnew;
        }
    }
    rc = leo_reconstruct_enqueue(enc, shards, present, size, recover_all);
    if (rc) return rc;
    RS_CUDA(cudaStreamSynchronize(enc->ctx->stream));
    if (written)
        for (int i = 0; i < end; i++)
            if (!present[i]) written[i] = 1;
    return RS_OK;
}

// leopard.go:393-419: re-encode into scratch and compare.
int leo_verify(rsgpu_encoder *enc, uint8_t *const *shards, size_t size, int *ok) {
    rsgpu_ctx *ctx = enc->ctx;
    if (size % 64) return RS_ERR_INVALID_SHARD_SIZE;
    const size_t pitch = (size + 255) & ~(size_t)255;
    int rc = ctx->scratch.ensure(pitch * (size_t)enc->p);
    if (rc) return rc;
    std::vector<uint8_t *> tmp(shards, shards + enc->total);
    for (int i = 0; i < enc->p; i++) tmp[enc->k + i] = ctx->scratch.ptr + pitch * i;
    rc = leo_encode_enqueue(enc, tmp.data(), size);
    if (rc) return rc;
    RS_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
    const uint8_t one = 1;
    for (int i = 0; i < enc->p; i++) {
        const uint8_t *src = tmp[enc->k + i];
        uint8_t *chk = shards[enc->k + i];
        RS_CUDA(launch_gf8_matmul(ctx->stream, ctx->info, &one, 1, 1, &src, &chk, size, kModeVerify, ctx->d_flag));
    }
    RS_CUDA(cudaMemcpyAsync(ctx->h_flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RS_CUDA(cudaStreamSynchronize(ctx->stream));
    *ok = (*ctx->h_flag == 0);
    return RS_OK;
}

}  // namespace rsgpu
