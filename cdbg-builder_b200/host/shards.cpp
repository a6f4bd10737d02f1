// Merging the outputs of a build split by bucket range across ranks (one GPU
// each).  No counterpart in the reference, which builds in one process.
//
// Rank r of G builds buckets [B*r/G, B*(r+1)/G) of the whole collection: its
// bucket records are exactly the single build's records of those buckets, so
// its fragments are the single build's fragments of those buckets, in the same
// order, except that their color-set ids are the rank's own (first appearance
// within its buckets).  The single build numbers color sets by first
// appearance over buckets 0..B-1, which is rank 0's classes in its order, then
// rank 1's classes that rank 0 did not have, and so on.  A class is its
// encoded bit string (the hybrid encoding of hybrid_color_sets.hpp:48-95 is a
// function of the set and the color count), so the merge deduplicates bit
// strings, appends each new one to the global bit vector, and rewrites the
// ids in the fragment records (unitig_spill.hpp:642-665 layout).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "cdbg_gpu.h"

namespace {

thread_local std::string t_err;

uint64_t get_bits(uint64_t const* w, uint64_t pos, uint32_t n) {  // n <= 64
    if (n == 0) return 0;
    const uint64_t i = pos >> 6;
    const uint32_t s = (uint32_t)(pos & 63);
    uint64_t v = w[i] >> s;
    if (s && s + n > 64) v |= w[i + 1] << (64 - s);
    return n == 64 ? v : (v & ((uint64_t(1) << n) - 1));
}

struct bit_appender {
    std::vector<uint64_t> w;
    uint64_t n = 0;
    void put(uint64_t v, uint32_t len) {  // len <= 64
        if (len == 0) return;
        if ((n >> 6) + 2 > w.size()) w.resize((n >> 6) + 2 + w.size() / 2, 0);
        const uint32_t s = (uint32_t)(n & 63);
        w[n >> 6] |= v << s;
        if (s && s + len > 64) w[(n >> 6) + 1] |= v >> (64 - s);
        n += len;
    }
};

// Bits [a, b) of a shard's words as whole words from bit 0 (the key of a class).
void extract(uint64_t const* w, uint64_t a, uint64_t b, std::vector<uint64_t>& out) {
    out.assign((b - a + 63) / 64, 0);
    for (uint64_t p = a, i = 0; p < b; p += 64, ++i) out[i] = get_bits(w, p, (uint32_t)std::min<uint64_t>(64, b - p));
}

uint64_t hash_words(std::vector<uint64_t> const& v, uint64_t nbits) {
    uint64_t h = 0x9E3779B97F4A7C15ULL ^ nbits;
    for (uint64_t x : v) {
        h ^= x + 0x9E3779B97F4A7C15ULL + (h << 6) + (h >> 2);
        h *= 0xff51afd7ed558ccdULL;
    }
    return h;
}

struct merged_out {
    std::vector<uint8_t> frag;
    std::vector<uint64_t> words;
    std::vector<uint64_t> offsets;
};

}  // namespace

extern "C" {

int cdbg_merge_shards(uint32_t num_shards, const uint8_t* const* frag, const uint64_t* frag_nbytes,
                      const uint64_t* const* class_words, const uint64_t* class_bits,
                      const uint64_t* const* class_offsets, const uint64_t* n_classes, cdbg_merged* out) {
    if (!out || (num_shards && (!frag || !frag_nbytes || !class_words || !class_bits || !class_offsets ||
                                !n_classes))) {
        t_err = "null argument";
        return -1;
    }
    try {
        auto* m = new merged_out();
        try {
            bit_appender gw;
            std::unordered_multimap<uint64_t, uint64_t> seen;  // key hash -> global id
            std::vector<uint64_t> key, other;
            uint64_t total_frag = 0;
            for (uint32_t s = 0; s < num_shards; ++s) total_frag += frag_nbytes[s];
            m->frag.reserve(total_frag);
            for (uint32_t s = 0; s < num_shards; ++s) {
                const uint64_t nc = n_classes[s];
                std::vector<uint64_t> map(nc);
                for (uint64_t c = 0; c < nc; ++c) {
                    const uint64_t a = class_offsets[s][c];
                    const uint64_t b = c + 1 < nc ? class_offsets[s][c + 1] : class_bits[s];
                    if (b < a || b > class_bits[s]) throw std::runtime_error("bad class offsets");
                    extract(class_words[s], a, b, key);
                    const uint64_t h = hash_words(key, b - a);
                    uint64_t gid = UINT64_MAX;
                    auto range = seen.equal_range(h);
                    for (auto it = range.first; it != range.second && gid == UINT64_MAX; ++it) {
                        const uint64_t g = it->second;
                        const uint64_t ga = m->offsets[g];
                        const uint64_t gb = g + 1 < m->offsets.size() ? m->offsets[g + 1] : gw.n;
                        if (gb - ga != b - a) continue;
                        extract(gw.w.data(), ga, gb, other);
                        if (other == key) gid = g;
                    }
                    if (gid == UINT64_MAX) {
                        gid = m->offsets.size();
                        m->offsets.push_back(gw.n);
                        for (uint64_t p = a; p < b; p += 64) {
                            const uint32_t len = (uint32_t)std::min<uint64_t>(64, b - p);
                            gw.put(get_bits(class_words[s], p, len), len);
                        }
                        seen.emplace(h, gid);
                    }
                    map[c] = gid;
                }
                // the shard's fragments with global ids
                const uint8_t* d = frag[s];
                const uint64_t n = frag_nbytes[s];
                uint64_t p = 0;
                while (p < n) {
                    if (p + 5 > n) throw std::runtime_error("truncated fragment record");
                    uint32_t nr;
                    std::memcpy(&nr, d + p + 1, 4);
                    const uint64_t q0 = m->frag.size();
                    const uint64_t rec_end_runs = p + 5 + 12ull * nr;
                    if (rec_end_runs + 4 > n) throw std::runtime_error("truncated fragment record");
                    uint32_t sl;
                    std::memcpy(&sl, d + rec_end_runs, 4);
                    const uint64_t end = rec_end_runs + 4 + sl;
                    if (end > n) throw std::runtime_error("truncated fragment record");
                    m->frag.insert(m->frag.end(), d + p, d + end);
                    for (uint32_t r = 0; r < nr; ++r) {
                        uint64_t cid;
                        std::memcpy(&cid, d + p + 5 + 12ull * r, 8);
                        if (cid != UINT64_MAX) {  // a foreign run keeps its marker
                            if (cid >= nc) throw std::runtime_error("fragment color-set id out of range");
                            const uint64_t g = map[cid];
                            std::memcpy(m->frag.data() + q0 + 5 + 12ull * r, &g, 8);
                        }
                    }
                    p = end;
                }
            }
            m->words.assign(gw.w.begin(), gw.w.begin() + (gw.n + 63) / 64);
            out->frag_bytes = m->frag.data();
            out->frag_nbytes = m->frag.size();
            out->class_words = m->words.data();
            out->class_bits = gw.n;
            out->class_offsets = m->offsets.data();
            out->n_color_sets = m->offsets.size();
            out->handle = m;
            return 0;
        } catch (...) {
            delete m;
            throw;
        }
    } catch (std::exception const& ex) {
        t_err = ex.what();
        return -1;
    }
}

void cdbg_merged_free(cdbg_merged* m) {
    if (!m || !m->handle) return;
    delete static_cast<merged_out*>(m->handle);
    m->handle = nullptr;
}

const char* cdbg_merge_last_error(void) { return t_err.c_str(); }

}  // extern "C"

// ---- phase 1 split by input file ---------------------------------------------
// Rank r reads its own slice of the input files (colors are global file
// indices) and runs phase 1 on it; the records of every bucket then go to the
// rank that owns the bucket, which merges the records all ranks made for it
// into the records one phase 1 over all the files makes.  That phase 1 orders
// a bucket's super-k-mer occurrences stably by the key (hash >> bb), in input
// order between equal keys, and merges runs of consecutive occurrences with
// equal key, length and bases (flags AND-ed, colors sorted unique).  Each
// rank's records are that list over its own occurrences, and the ranks' files
// are consecutive slices of the input, so the stable order of all the ranks'
// records taken in rank order, merged the same way, is the one over all the
// occurrences: merging runs of equal neighbours is the same whether done at
// once or first within each rank's stretch.
namespace {

// The 64-bit key hash of a super-k-mer (length, then its 2-bit bases 32 at a
// time, base i at bits 2(i%32) of word i/32, unused bits zero): the hash
// phase 1 sorts by.
uint64_t mix64_host(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

uint64_t super_hash_packed(uint8_t const* packed, uint32_t len) {
    uint64_t h = mix64_host(0x51ed2701f3a5c2b9ULL ^ (uint64_t)len);
    const uint64_t nb = ((uint64_t)len + 3) / 4;
    for (uint64_t i = 0; i < nb; i += 8) {
        uint64_t w = 0;
        std::memcpy(&w, packed + i, (size_t)std::min<uint64_t>(8, nb - i));
        h = mix64_host(h ^ w);
    }
    return h;
}

bool get_varint(uint8_t const* b, uint64_t end, uint64_t& p, uint64_t& v) {
    v = 0;
    for (uint32_t sh = 0; p < end && sh < 64; sh += 7) {
        const uint8_t c = b[p++];
        v |= (uint64_t)(c & 0x7f) << sh;
        if (!(c & 0x80)) return true;
    }
    return false;
}

void put_varint(uint64_t v, std::vector<uint8_t>& out) {
    while (v >= 0x80) {
        out.push_back((uint8_t)(v | 0x80));
        v >>= 7;
    }
    out.push_back((uint8_t)v);
}

// One serialized bucket record (super_kmer.hpp:105-143 layout: varint color
// count, varint color gaps, varint (len << 4 | flags), 2-bit bases).
struct rec_ref {
    uint64_t key;
    uint32_t len, flags;
    uint8_t const* bases;
    std::vector<uint32_t> colors;
};

void parse_records(uint8_t const* b, uint64_t n, uint32_t bb, std::vector<rec_ref>& out) {
    uint64_t p = 0;
    while (p < n) {
        rec_ref r;
        uint64_t nc, v;
        if (!get_varint(b, n, p, nc)) throw std::runtime_error("malformed bucket record");
        r.colors.resize(nc);
        uint32_t prev = 0;
        for (uint64_t c = 0; c < nc; ++c) {
            if (!get_varint(b, n, p, v)) throw std::runtime_error("malformed bucket record");
            prev += (uint32_t)v;
            r.colors[c] = prev;
        }
        if (!get_varint(b, n, p, v)) throw std::runtime_error("malformed bucket record");
        r.len = (uint32_t)(v >> 4);
        r.flags = (uint32_t)(v & 0xf);
        const uint64_t pb = ((uint64_t)r.len + 3) / 4;
        if (p + pb > n) throw std::runtime_error("malformed bucket record");
        r.bases = b + p;
        p += pb;
        const uint64_t h = super_hash_packed(r.bases, r.len);
        r.key = bb ? (h >> bb) : h;
        out.push_back(std::move(r));
    }
}

struct merged_records_out {
    std::vector<uint8_t> bytes;
    std::vector<uint64_t> off;
};

}  // namespace

extern "C" {

int cdbg_merge_bucket_records(uint32_t num_sources, const uint8_t* const* src, const uint64_t* const* src_off,
                              uint32_t num_buckets, uint32_t b_lo, uint32_t b_hi, cdbg_merged_records* out) {
    try {
        if (!out || (num_sources && (!src || !src_off))) throw std::runtime_error("null argument");
        if (b_lo > b_hi || b_hi > num_buckets) throw std::runtime_error("bad bucket range");
        uint32_t bb = 0;
        while ((1ull << bb) < num_buckets) ++bb;
        auto* m = new merged_records_out();
        try {
            const uint32_t nb = b_hi - b_lo;
            m->off.assign(nb + 1, 0);
            std::vector<rec_ref> recs;
            std::vector<uint32_t> idx;
            for (uint32_t i = 0; i < nb; ++i) {
                recs.clear();
                for (uint32_t s = 0; s < num_sources; ++s)
                    parse_records(src[s] + src_off[s][i], src_off[s][i + 1] - src_off[s][i], bb, recs);
                idx.resize(recs.size());
                for (uint32_t j = 0; j < idx.size(); ++j) idx[j] = j;
                std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return recs[a].key < recs[b].key; });
                size_t j = 0;
                while (j < idx.size()) {
                    rec_ref const& a = recs[idx[j]];
                    std::vector<uint32_t> colors = a.colors;
                    uint32_t flags = a.flags;
                    size_t t = j + 1;
                    for (; t < idx.size(); ++t) {
                        rec_ref const& c = recs[idx[t]];
                        if (c.key != a.key || c.len != a.len ||
                            std::memcmp(c.bases, a.bases, ((size_t)a.len + 3) / 4) != 0)
                            break;
                        flags &= c.flags;
                        colors.insert(colors.end(), c.colors.begin(), c.colors.end());
                    }
                    if (t > j + 1) {
                        std::sort(colors.begin(), colors.end());
                        colors.erase(std::unique(colors.begin(), colors.end()), colors.end());
                    }
                    put_varint(colors.size(), m->bytes);
                    uint32_t prev = 0;
                    for (uint32_t c : colors) {
                        put_varint(c - prev, m->bytes);
                        prev = c;
                    }
                    put_varint(((uint64_t)a.len << 4) | flags, m->bytes);
                    m->bytes.insert(m->bytes.end(), a.bases, a.bases + ((size_t)a.len + 3) / 4);
                    j = t;
                }
                m->off[i + 1] = m->bytes.size();
            }
            out->bytes = m->bytes.data();
            out->nbytes = m->bytes.size();
            out->bucket_off = m->off.data();
            out->handle = m;
            return 0;
        } catch (...) {
            delete m;
            throw;
        }
    } catch (std::exception const& ex) {
        t_err = ex.what();
        return -1;
    }
}

int cdbg_class_strings(const uint64_t* words, uint64_t class_bits, const uint64_t* offsets, uint64_t n,
                       uint64_t* hashes, uint64_t* strings, uint64_t strings_cap, uint64_t* string_off) {
    try {
        if (n && (!words || !offsets || !hashes || !string_off)) throw std::runtime_error("null argument");
        std::vector<uint64_t> key;
        uint64_t at = 0;
        string_off[0] = 0;
        for (uint64_t c = 0; c < n; ++c) {
            const uint64_t a = offsets[c], b = c + 1 < n ? offsets[c + 1] : class_bits;
            if (b < a || b > class_bits) throw std::runtime_error("bad class offsets");
            extract(words, a, b, key);
            hashes[c] = hash_words(key, b - a);
            if (at + key.size() > strings_cap) throw std::runtime_error("class strings buffer too small");
            if (!key.empty()) std::memcpy(strings + at, key.data(), 8 * key.size());
            at += key.size();
            string_off[c + 1] = at;
        }
        return 0;
    } catch (std::exception const& ex) {
        t_err = ex.what();
        return -1;
    }
}

int cdbg_frag_remap_classes(uint8_t* frag, uint64_t n, const uint64_t* map, uint64_t nmap) {
    try {
        if (n && (!frag || (nmap && !map))) throw std::runtime_error("null argument");
        uint64_t p = 0;
        while (p < n) {
            if (p + 5 > n) throw std::runtime_error("truncated fragment record");
            uint32_t nr;
            std::memcpy(&nr, frag + p + 1, 4);
            const uint64_t runs_end = p + 5 + 12ull * nr;
            if (runs_end + 4 > n) throw std::runtime_error("truncated fragment record");
            uint32_t sl;
            std::memcpy(&sl, frag + runs_end, 4);
            if (runs_end + 4 + sl > n) throw std::runtime_error("truncated fragment record");
            for (uint32_t r = 0; r < nr; ++r) {
                uint64_t cid;
                std::memcpy(&cid, frag + p + 5 + 12ull * r, 8);
                if (cid == UINT64_MAX) continue;  // a foreign run keeps its marker
                if (cid >= nmap) throw std::runtime_error("fragment color-set id out of range");
                std::memcpy(frag + p + 5 + 12ull * r, map + cid, 8);
            }
            p = runs_end + 4 + sl;
        }
        return 0;
    } catch (std::exception const& ex) {
        t_err = ex.what();
        return -1;
    }
}

void cdbg_merged_records_free(cdbg_merged_records* m) {
    if (!m || !m->handle) return;
    delete static_cast<merged_records_out*>(m->handle);
    m->handle = nullptr;
}

}  // extern "C"
