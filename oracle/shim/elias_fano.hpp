#pragma once
// Clean-room stand-in for `bits::elias_fano<false,false>` (test
// infrastructure only; the reference's `external/bits` submodule is absent).
// The reference only encodes the per-class bit offsets with it at
// streaming_color_set_dict.hpp:253-269 and serializes it with
// essentials::generic_saver.  Textbook Elias-Fano: l = floor(log2(U/n)) low
// bits per value stored verbatim, high parts as a unary-coded bit vector of
// n + (U >> l) + 1 bits with bit (x_i >> l) + i set.

#include <cstdint>
#include <vector>

#include "bit_vector.hpp"

namespace bits {

template <bool index_zeros = false, bool encode_prefix_sum = false>
struct elias_fano {
    template <typename Iterator>
    void encode(Iterator begin, uint64_t n, uint64_t universe) {
        m_num_values = n;
        m_universe = universe;
        m_l = 0;
        if (n > 0 && universe > n) {
            uint64_t q = universe / n;
            while ((uint64_t(1) << (m_l + 1)) <= q) ++m_l;
        }
        bit_vector::builder low, high;
        high.resize(n + (universe >> m_l) + 1);
        for (uint64_t i = 0; i < n; ++i, ++begin) {
            const uint64_t x = *begin;
            if (m_l) low.append_bits(x, m_l);
            high.set((x >> m_l) + i);
        }
        low.build(m_low);
        high.build(m_high);
    }

    uint64_t size() const { return m_num_values; }

    // Linear-time access; used only by tests of the shim itself.
    uint64_t access(uint64_t i) const {
        uint64_t seen = 0, pos = 0;
        auto const& w = m_high.data();
        for (uint64_t wi = 0; wi < w.size(); ++wi) {
            uint64_t word = w[wi];
            while (word) {
                const uint64_t b = (uint64_t)__builtin_ctzll(word);
                pos = wi * 64 + b;
                if (seen == i) {
                    const uint64_t hi = pos - i;
                    uint64_t lo = 0;
                    if (m_l) {
                        bit_vector::iterator it(m_low.data().data(), m_low.data().size(), i * m_l);
                        lo = it.take(m_l);
                    }
                    return (hi << m_l) | lo;
                }
                ++seen;
                word &= word - 1;
            }
        }
        return 0;
    }

    template <typename Visitor>
    void visit(Visitor& v) {
        v.visit(m_universe);
        v.visit(m_num_values);
        v.visit(m_l);
        v.visit(m_low);
        v.visit(m_high);
    }

private:
    uint64_t m_universe = 0;
    uint64_t m_num_values = 0;
    uint64_t m_l = 0;
    bit_vector m_low;
    bit_vector m_high;
};

}  // namespace bits
