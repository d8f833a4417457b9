// gf8_device.cuh -- device helpers of the GF(2^8) contraction, shared by the
// per-call kernels (kernels_gf8.cu) and the batched kernel (batch.cu).
#pragma once

#include "kernels.h"

namespace rsgpu {
namespace gf8dev {

constexpr int kThreads = 256;
constexpr int kHalfStride = 256;         // bytes between the tables of one (input, half)
constexpr int kInStride = 2 * kHalfStride;
constexpr int kTableAlign = 256;         // table base alignment in the shared window

// GF(2^8) product, polynomial 0x11D, by shift-and-add (unique field product,
// identical to galMultiply's table).
__device__ __forceinline__ uint32_t gf_mul_dev(uint32_t a, uint32_t b) {
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        r ^= (b & 1u) ? a : 0u;
        b >>= 1;
        a = (a << 1) ^ ((a & 0x80u) ? 0x11Du : 0u);
    }
    return r & 0xFFu;
}

// Shared table layout: word (i*2 + h)*64 + g*16 + e; the entry's byte o is
// coef[4g+o][i] * (e << 4h) (zero for o >= n_out).
template <int G>
__device__ __forceinline__ void build_tables_from(uint32_t *tab, const uint8_t (*coef)[kMaxIn], int n_in,
                                                  int n_out) {
    const int total = n_in * 2 * G * 16;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int e = w & 15;
        const int g = (w >> 4) % G;
        const int ih = (w >> 4) / G;
        const int h = ih & 1, i = ih >> 1;
        const uint32_t x = (uint32_t)e << (4 * h);
        uint32_t word = 0;
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const int oo = 4 * g + o;
            if (oo < n_out) word |= gf_mul_dev(coef[oo][i], x) << (8 * o);
        }
        tab[ih * (kHalfStride / 4) + g * 16 + e] = word;
    }
}

template <int G>
__device__ __forceinline__ void build_tables(uint32_t *tab, const GfMatArgs &a) {
    build_tables_from<G>(tab, a.coef, a.n_in, a.n_out);
}

__device__ __forceinline__ uint32_t *aligned_tables(uint32_t *raw) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(raw);
    const uint32_t pad = ((s + (kTableAlign - 1)) & ~(uint32_t)(kTableAlign - 1)) - s;
    return raw + pad / 4;
}

__device__ __forceinline__ uint32_t lds(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ uint32_t mulhi(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

__device__ __forceinline__ uint32_t madhi(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}

struct Mul {
    uint32_t m[8];
};

// Shared addresses of the 8 nibble lookups of word x (lo[j], hi[j] for byte j).
// lb/hb: table bases of this input, 256-byte aligned.
template <int V>
__device__ __forceinline__ void nibble_addrs(uint32_t x, uint32_t lb, uint32_t hb, const Mul &mu,
                                             uint32_t (&l)[4], uint32_t (&h)[4]) {
    if (V == kVariantShift) {
        l[0] = ((x << 2) & 0x3Cu) | lb;  h[0] = ((x >> 2) & 0x3Cu) | hb;
        l[1] = ((x >> 6) & 0x3Cu) | lb;  h[1] = ((x >> 10) & 0x3Cu) | hb;
        l[2] = ((x >> 14) & 0x3Cu) | lb; h[2] = ((x >> 18) & 0x3Cu) | hb;
        l[3] = ((x >> 22) & 0x3Cu) | lb; h[3] = ((x >> 26) & 0x3Cu) | hb;
    } else if (V == kVariantMulHi) {
        l[0] = ((x * mu.m[0]) & 0x3Cu) | lb;
        l[1] = (mulhi(x, mu.m[1]) & 0x3Cu) | lb;
        l[2] = (mulhi(x, mu.m[2]) & 0x3Cu) | lb;
        l[3] = (mulhi(x, mu.m[3]) & 0x3Cu) | lb;
        h[0] = (mulhi(x, mu.m[4]) & 0x3Cu) | hb;
        h[1] = (mulhi(x, mu.m[5]) & 0x3Cu) | hb;
        h[2] = (mulhi(x, mu.m[6]) & 0x3Cu) | hb;
        h[3] = (mulhi(x, mu.m[7]) & 0x3Cu) | hb;
    } else {
        // bytes of lo4/hi4 are 4*nibble; PRMT drops byte j into the (zero)
        // low byte of the 256-aligned table base.  Byte 3 goes through the
        // FMA pipe instead (hi32(v * 256) + base), which takes a quarter of
        // the address work off the integer ALU pipe.
        const uint32_t lo4 = (x * mu.m[0]) & 0x3C3C3C3Cu;
        const uint32_t hi4 = mulhi(x, mu.m[4]) & 0x3C3C3C3Cu;
        l[0] = __byte_perm(lo4, lb, 0x7650); h[0] = __byte_perm(hi4, hb, 0x7650);
        l[1] = __byte_perm(lo4, lb, 0x7651); h[1] = __byte_perm(hi4, hb, 0x7651);
        l[2] = __byte_perm(lo4, lb, 0x7652); h[2] = __byte_perm(hi4, hb, 0x7652);
        l[3] = madhi(lo4, 256u, lb);         h[3] = madhi(hi4, 256u, hb);
    }
}

// acc[g][P..P+3] ^= products of the 4 bytes of x.
template <int G, int P, int V>
__device__ __forceinline__ void mac_word(uint32_t x, uint32_t lb, const Mul &mu, uint32_t (&acc)[G][16]) {
    uint32_t l[4], h[4];
    nibble_addrs<V>(x, lb, lb + kHalfStride, mu, l, h);
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[g][P + j] ^= lds(l[j] + 64 * g) ^ lds(h[j] + 64 * g);
}

template <int G, int V>
__device__ __forceinline__ void mac_vec(const uint4 &x, uint32_t lb, const Mul &mu, uint32_t (&acc)[G][16]) {
    mac_word<G, 0, V>(x.x, lb, mu, acc);
    mac_word<G, 4, V>(x.y, lb, mu, acc);
    mac_word<G, 8, V>(x.z, lb, mu, acc);
    mac_word<G, 12, V>(x.w, lb, mu, acc);
}

// a_b holds output bytes [o0..o3] of position b; returns per-output words.
__device__ __forceinline__ void transpose4x4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                             uint32_t &o0, uint32_t &o1, uint32_t &o2, uint32_t &o3) {
    const uint32_t t0 = __byte_perm(a0, a1, 0x5140), t1 = __byte_perm(a2, a3, 0x5140);
    const uint32_t t2 = __byte_perm(a0, a1, 0x7362), t3 = __byte_perm(a2, a3, 0x7362);
    o0 = __byte_perm(t0, t1, 0x5410);
    o1 = __byte_perm(t0, t1, 0x7632);
    o2 = __byte_perm(t2, t3, 0x5410);
    o3 = __byte_perm(t2, t3, 0x7632);
}

__device__ __forceinline__ uint4 ld_in(const uint8_t *p, long long v) {
    return __ldcs(reinterpret_cast<const uint4 *>(p) + v);
}


}  // namespace gf8dev
}  // namespace rsgpu
