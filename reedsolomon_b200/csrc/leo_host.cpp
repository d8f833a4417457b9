// leo_host.cpp -- Leopard field tables and error locators on the host.
#include "leo_host.h"

namespace rsgpu {
namespace {

// Cantor bases (leopard.go:1105-1110, leopard8.go:1030-1032) and generator
// polynomials (leopard.go:104, leopard8.go:101).
const uint16_t kCantor16[16] = {0x0001, 0xACCA, 0x3C0E, 0x163E, 0xC582, 0xED2E, 0x914C, 0x4012,
                                0x6C98, 0x10D8, 0x6A72, 0xB900, 0xFDB8, 0xFB34, 0xFF38, 0x991E};
const uint16_t kCantor8[8] = {1, 214, 152, 146, 86, 200, 88, 230};

template <int BITS>
inline uint16_t add_mod(uint16_t a, uint16_t b) {
    // partial reduction, may return the modulus (leopard.go:1001-1006)
    uint64_t s = (uint64_t)a + b;
    return (uint16_t)((s + (s >> BITS)) & ((1u << BITS) - 1));
}

template <int BITS>
inline uint16_t sub_mod(uint16_t a, uint16_t b) {
    uint64_t d = (uint64_t)a - (uint64_t)b;  // wraps like Go's uint
    return (uint16_t)((d + (d >> BITS)) & ((1u << BITS) - 1));
}

// Walsh-Hadamard transform mod (2^BITS - 1), radix-4 groups starting below
// mtrunc only (leopard.go:1025-1060).
template <int BITS>
void fwht(uint16_t *data, unsigned mtrunc) {
    const unsigned order = 1u << BITS;
    for (unsigned dist = 1, dist4 = 4; dist4 <= order; dist = dist4, dist4 <<= 2)
        for (unsigned r = 0; r < mtrunc; r += dist4)
            for (unsigned i = r; i < r + dist; i++) {
                uint16_t t0 = data[i], t1 = data[i + dist], t2 = data[i + 2 * dist], t3 = data[i + 3 * dist];
                uint16_t a = add_mod<BITS>(t0, t1), b = sub_mod<BITS>(t0, t1);
                uint16_t c = add_mod<BITS>(t2, t3), d = sub_mod<BITS>(t2, t3);
                data[i] = add_mod<BITS>(a, c);
                data[i + 2 * dist] = sub_mod<BITS>(a, c);
                data[i + dist] = add_mod<BITS>(b, d);
                data[i + 3 * dist] = sub_mod<BITS>(b, d);
            }
}

}  // namespace

template <int BITS>
uint16_t LeoField<BITS>::mul_log(uint16_t a, uint16_t log_b) const {
    if (a == 0) return 0;
    return exp[add_mod<BITS>(log[a], log_b)];
}

template <int BITS>
LeoField<BITS>::LeoField() : log(kOrder), exp(kOrder), skew(kMod), walsh(kOrder) {
    const unsigned poly = BITS == 16 ? 0x1002D : 0x11D;
    const uint16_t *cantor = BITS == 16 ? kCantor16 : kCantor8;
    // LFSR powers (exp stores the exponent of each element here), then the
    // Cantor-basis element -> exponent map, then its inverse.
    unsigned state = 1;
    for (unsigned i = 0; i < kMod; i++) {
        exp[state] = (uint16_t)i;
        state <<= 1;
        if (state >= kOrder) state ^= poly;
    }
    exp[0] = (uint16_t)kMod;
    log[0] = 0;
    for (int i = 0; i < BITS; i++) {
        const unsigned width = 1u << i;
        for (unsigned j = 0; j < width; j++) log[j + width] = log[j] ^ cantor[i];
    }
    for (unsigned i = 0; i < kOrder; i++) log[i] = exp[log[i]];
    for (unsigned i = 0; i < kOrder; i++) exp[log[i]] = (uint16_t)i;
    exp[kMod] = exp[0];

    // FFT skew factors (leopard.go:1150-1195)
    std::vector<uint16_t> temp(BITS - 1);
    for (int i = 1; i < BITS; i++) temp[i - 1] = (uint16_t)(1u << i);
    for (int m = 0; m < BITS - 1; m++) {
        const unsigned step = 1u << (m + 1);
        skew[(1u << m) - 1] = 0;
        for (int i = m; i < BITS - 1; i++) {
            const unsigned s = 1u << (i + 1);
            for (unsigned j = (1u << m) - 1; j < s; j += step) skew[j + s] = skew[j] ^ temp[i];
        }
        temp[m] = (uint16_t)(kMod - log[mul_log(temp[m], log[temp[m] ^ 1])]);
        for (int i = m + 1; i < BITS - 1; i++) {
            const uint16_t sum = add_mod<BITS>(log[temp[i] ^ 1], temp[m]);
            temp[i] = mul_log(temp[i], sum);
        }
    }
    for (unsigned i = 0; i < kMod; i++) skew[i] = log[skew[i]];
    for (unsigned i = 0; i < kOrder; i++) walsh[i] = log[i];
    walsh[0] = 0;
    fwht<BITS>(walsh.data(), kOrder);
}

template <int BITS>
const LeoField<BITS> &LeoField<BITS>::get() {
    static const LeoField<BITS> f;
    return f;
}

template struct LeoField<16>;
template struct LeoField<8>;

}  // namespace rsgpu
