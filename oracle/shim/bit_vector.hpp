#pragma once
// Clean-room stand-in for the `bits::bit_vector` API the reference uses
// (test infrastructure only: it lets oracle/Makefile compile the reference
// from its own sources).  The reference's `external/bits` submodule is absent
// from this checkout, so the layout here is this project's definition, written
// from the API surface the reference calls:
//   builder: append_bits, append, resize, set, get_word64, num_bits, data,
//            clear, build      (compact_color_set_dict.hpp:81-155,
//                               hybrid_color_sets.hpp:62-65,
//                               streaming_color_set_dict.hpp:160-364)
//   iterator(words, num_words, pos), take(n)   (compact_color_set_dict.hpp:100,193)
// Bits are stored LSB-first in 64-bit little-endian words: bit i of the
// vector is bit (i % 64) of word (i / 64).  Unused high bits of the last word
// are kept at zero.  The same convention is used by the GPU color-set writer,
// so .color_sets words are comparable byte for byte between the two.

#include <cassert>
#include <cstdint>
#include <vector>

namespace bits {

struct bit_vector {
    struct builder {
        builder() = default;

        void clear() {
            m_data.clear();
            m_num_bits = 0;
        }

        // Append the low `len` bits of `x` (len <= 64).
        void append_bits(uint64_t x, uint64_t len) {
            assert(len <= 64);
            if (len == 0) return;
            if (len < 64) x &= (uint64_t(1) << len) - 1;
            const uint64_t off = m_num_bits & 63;
            if (off == 0) {
                m_data.push_back(x);
            } else {
                m_data.back() |= x << off;
                if (off + len > 64) m_data.push_back(x >> (64 - off));
            }
            m_num_bits += len;
        }

        void append(builder const& other) {
            const uint64_t n = other.m_num_bits;
            uint64_t pos = 0;
            while (pos < n) {
                const uint64_t take = (n - pos) < 64 ? (n - pos) : 64;
                append_bits(other.get_word64(pos), take);
                pos += take;
            }
        }

        // Grow (or shrink) to n bits; new bits are zero.
        void resize(uint64_t n) {
            m_data.resize((n + 63) / 64, 0);
            if (n & 63) m_data.back() &= (uint64_t(1) << (n & 63)) - 1;
            m_num_bits = n;
        }

        void set(uint64_t pos, bool b = true) {
            assert(pos < m_num_bits);
            const uint64_t w = pos >> 6, s = pos & 63;
            if (b)
                m_data[w] |= uint64_t(1) << s;
            else
                m_data[w] &= ~(uint64_t(1) << s);
        }

        // 64 bits starting at bit `pos`; positions past num_bits read as 0.
        uint64_t get_word64(uint64_t pos) const {
            const uint64_t w = pos >> 6, s = pos & 63;
            if (w >= m_data.size()) return 0;
            uint64_t lo = m_data[w] >> s;
            if (s != 0 && w + 1 < m_data.size()) lo |= m_data[w + 1] << (64 - s);
            return lo;
        }

        uint64_t num_bits() const { return m_num_bits; }
        std::vector<uint64_t>& data() { return m_data; }
        std::vector<uint64_t> const& data() const { return m_data; }

        void build(bit_vector& bv) {
            bv.m_num_bits = m_num_bits;
            bv.m_data.swap(m_data);
            clear();
        }

    private:
        std::vector<uint64_t> m_data;
        uint64_t m_num_bits = 0;
    };

    struct iterator {
        iterator() = default;
        iterator(uint64_t const* data, uint64_t num_words, uint64_t pos = 0)
            : m_data(data), m_num_words(num_words), m_pos(pos) {}

        // Read the next n bits (n <= 64), LSB-first.
        uint64_t take(uint64_t n) {
            if (n == 0) return 0;
            const uint64_t v = peek64_();
            m_pos += n;
            return n == 64 ? v : (v & ((uint64_t(1) << n) - 1));
        }

        // Advance past a run of zero bits and return its length; the cursor
        // then sits on the terminating one bit (not consumed).
        uint64_t skip_zeros() {
            uint64_t zeros = 0;
            for (;;) {
                const uint64_t v = peek64_();
                if (v != 0) {
                    const uint64_t z = (uint64_t)__builtin_ctzll(v);
                    zeros += z;
                    m_pos += z;
                    return zeros;
                }
                zeros += 64;
                m_pos += 64;
                if ((m_pos >> 6) > m_num_words) return zeros;  // ran off the end
            }
        }

        uint64_t position() const { return m_pos; }

    private:
        uint64_t peek64_() const {
            const uint64_t w = m_pos >> 6, s = m_pos & 63;
            if (!m_data || w >= m_num_words) return 0;
            uint64_t lo = m_data[w] >> s;
            if (s != 0 && w + 1 < m_num_words) lo |= m_data[w + 1] << (64 - s);
            return lo;
        }
        uint64_t const* m_data = nullptr;
        uint64_t m_num_words = 0;
        uint64_t m_pos = 0;
    };

    uint64_t num_bits() const { return m_num_bits; }
    std::vector<uint64_t> const& data() const { return m_data; }

    template <typename Visitor>
    void visit(Visitor& v) {
        v.visit(m_num_bits);
        v.visit(m_data);
    }
    template <typename Visitor>
    void visit(Visitor& v) const {
        v.visit(m_num_bits);
        v.visit(m_data);
    }

private:
    uint64_t m_num_bits = 0;
    std::vector<uint64_t> m_data;
};

}  // namespace bits
