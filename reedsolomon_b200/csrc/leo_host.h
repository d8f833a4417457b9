// leo_host.h -- host-side Leopard field tables and error locators.
//
// Restates the table construction of leopard.go:1104-1274 (GF(2^16)) and
// leopard8.go:1029-1137 (GF(2^8)).  The per-pattern error locators are
// computed on the device (leo_errloc_kernel in leopard.cu).
#pragma once

#include <cstdint>
#include <vector>

namespace rsgpu {

template <int BITS>
struct LeoField {
    static constexpr unsigned kOrder = 1u << BITS;
    static constexpr unsigned kMod = kOrder - 1;
    std::vector<uint16_t> log, exp;   // Cantor-basis log / exp (kOrder entries)
    std::vector<uint16_t> skew;       // fftSkew (kMod entries)
    std::vector<uint16_t> walsh;      // FWHT(log) (kOrder entries)
    static const LeoField &get();
    uint16_t mul_log(uint16_t a, uint16_t log_b) const;

  private:
    LeoField();
};

using Leo16 = LeoField<16>;
using Leo8 = LeoField<8>;

inline unsigned ceil_pow2(unsigned n) {
    unsigned r = 1;
    while (r < n) r <<= 1;
    return r;
}

}  // namespace rsgpu
