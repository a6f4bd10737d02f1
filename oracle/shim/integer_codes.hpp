#pragma once
// Clean-room stand-in for `bits::util::write_delta` / `read_delta`
// (test infrastructure only; the reference's `external/bits` submodule is
// absent).  The reference calls write_delta on values that may be zero
// (hybrid_color_sets.hpp:51-87: a set size, a first color, a gap), so this
// definition codes x >= 0 as the Elias delta code of y = x + 1:
//
//   gamma(y), y >= 1:  l = floor(log2 y); emit l zero bits, one 1 bit, then the
//                      low l bits of y (LSB-first, as bit_vector::append_bits).
//   delta(x):          y = x + 1; l = floor(log2 y); emit gamma(l + 1), then the
//                      low l bits of y.
//
// The GPU color-set encoder implements the same definition, so both produce
// the same .color_sets words.  Whether this matches the upstream `bits`
// library bit for bit cannot be checked here (the submodule is absent).

#include <cstdint>

#include "bit_vector.hpp"

namespace bits {
namespace util {

inline uint64_t msb_(uint64_t y) { return 63u - (uint64_t)__builtin_clzll(y); }

inline void append_zeros_(bit_vector::builder& b, uint64_t n) {
    while (n >= 64) {
        b.append_bits(0, 64);
        n -= 64;
    }
    if (n) b.append_bits(0, n);
}

inline void write_gamma(bit_vector::builder& b, uint64_t y) {
    const uint64_t l = msb_(y);
    append_zeros_(b, l);
    b.append_bits(1, 1);
    if (l) b.append_bits(y, l);  // append_bits masks to the low l bits
}

inline void write_delta(bit_vector::builder& b, uint64_t x) {
    const uint64_t y = x + 1;
    const uint64_t l = msb_(y);
    write_gamma(b, l + 1);
    if (l) b.append_bits(y, l);
}

template <typename Iterator>
inline uint64_t read_gamma(Iterator& it) {
    const uint64_t l = it.skip_zeros();
    it.take(1);
    const uint64_t low = l ? it.take(l) : 0;
    return (l >= 64 ? 0 : (uint64_t(1) << l)) | low;
}

template <typename Iterator>
inline uint64_t read_delta(Iterator& it) {
    const uint64_t l = read_gamma(it) - 1;
    const uint64_t low = l ? it.take(l) : 0;
    return ((uint64_t(1) << l) | low) - 1;
}

}  // namespace util
}  // namespace bits
