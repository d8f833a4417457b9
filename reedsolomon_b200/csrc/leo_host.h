// leo_host.h -- host-side Leopard field tables and error locators.
//
// Restates the table construction of leopard.go:1104-1274 (GF(2^16)) and
// leopard8.go:1029-1137 (GF(2^8)) and the error-locator evaluation of
// leopard.go:468-510 / leopard8.go:434-513, which stays on the host (FWHT over
// the field order per erasure pattern, cached per pattern).
#pragma once

#include <cstdint>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
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

// Error locators for an erasure pattern (present[k+p]); returns kOrder values.
// Cached per pattern (bounded LRU) like leopard8.go's inversion map.
class ErrLocCache {
  public:
    explicit ErrLocCache(size_t capacity = 256) : cap_(capacity) {}
    std::shared_ptr<const std::vector<uint16_t>> get(int bits, int k, int p, const uint8_t *present);

  private:
    using Entry = std::shared_ptr<const std::vector<uint16_t>>;
    size_t cap_;
    std::mutex mu_;
    std::list<std::string> lru_;
    std::map<std::string, std::pair<Entry, std::list<std::string>::iterator>> map_;
};

std::vector<uint16_t> leo_errlocs(int bits, int k, int p, const uint8_t *present);

inline unsigned ceil_pow2(unsigned n) {
    unsigned r = 1;
    while (r < n) r <<= 1;
    return r;
}

}  // namespace rsgpu
