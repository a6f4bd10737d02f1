// ORACLE -- CPU restatement of the reference's phase 1 (bucket-write) and
// phase 2 (bucket-process) for parity testing.  TEST INFRASTRUCTURE ONLY:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load it, as a checker; the shipped GPU path never calls it.
//
// Parity pin: outputs of this file are checked against the reference's own
// code built from its unmodified sources (oracle/Makefile -> oracle/_ref/:
// ref_phase1 = bucket_ingester.hpp's ingest_file_bucketed, ref_phase2 =
// bucket_walker.hpp's process_buckets, cdbg-build = the whole pipeline, which
// passes the reference's test_data/verify.py on salmonella_10), and the
// committed fixtures under tests/golden/ were produced by those binaries.
//
// Function map (reference file:line each restates):
//   nt_seed/rol/ror, nthash_init, nthash_roll -> phase1_bucket_write/minimizer.hpp:21-62
//   compute_best_m                           -> minimizer.hpp:65-73
//   min_scan (windowed minimum, <= ties)     -> minimizer.hpp:94-157
//   emit_supers                              -> bucket_ingester.hpp:36-127
//   read_sequences / acgt runs               -> seq_reader.hpp:66 + kseq.h,
//                                               bucket_ingester.hpp:129-177, kmer.hpp:35
//   pack / varint / record layout            -> super_kmer.hpp:43-143
//   frames                                   -> bucket_io.hpp:19-40,201-277,651-705
//   process_bucket (load/resolve/walk)       -> bucket_walker.hpp:166-570
//   merge into the global dict (T = 1)       -> bucket_walker.hpp:713-761,
//                                               streaming_color_set_dict.hpp:148-182
//   hybrid encoding                          -> hybrid_color_sets.hpp:48-95
//   frag record layout                       -> unitig_spill.hpp:491-522
//   .color_sets finalize layout              -> streaming_color_set_dict.hpp:221-294
//
// The canonical bucket-record order (full per-bucket dedup, records ordered
// by (bucket, 64-bit key hash) with input order kept among equal hashes) is
// this project's GPU phase-1 output order; the oracle reproduces it so bucket
// files can be compared byte for byte after LZ4 decompression.

#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

extern "C" {
int LZ4_compressBound(int inputSize);
int LZ4_compress_default(const char* src, char* dst, int srcSize, int dstCapacity);
int LZ4_decompress_safe(const char* src, char* dst, int compressedSize, int dstCapacity);
}

namespace oracle {

typedef unsigned __int128 u128;

// ---------------------------------------------------------------- k-mers
template <typename K>
K kmask(uint32_t k) {
    if (2 * k >= sizeof(K) * 8) return ~K(0);
    return (K(1) << (2 * k)) - 1;
}

// Reverse complement by reversing 2-bit groups (kmer.hpp:80-106 computes the
// same function with SWAR steps; this is the plain loop).
template <typename K>
K revcomp(K x, uint32_t k) {
    K r = 0;
    for (uint32_t i = 0; i < k; ++i) {
        r = (r << 2) | (K)(3 - (uint32_t)(x & 3));
        x >>= 2;
    }
    return r;
}

template <typename K>
K canon(K x, uint32_t k) {
    K r = revcomp(x, k);
    return x <= r ? x : r;
}

// ---------------------------------------------------------------- ntHash
static const uint64_t NT[4] = {0x3c8bfbb395c60474ULL, 0x3193c18562a02b4cULL,
                               0x20323ed082572324ULL, 0x295549f54be24456ULL};
inline uint64_t rol(uint64_t x, unsigned r) {
    r &= 63;
    return r ? (x << r) | (x >> (64 - r)) : x;
}

// Canonical ntHash of the m-mer at s, computed directly (no rolling):
// fwd = XOR_i rol(NT[s_i], m-1-i); rc = XOR_i rol(NT[3 - s_{m-1-i}], m-1-i).
// Equal to the rolled values of minimizer.hpp:40-62 because rol distributes
// over XOR.
inline uint64_t canon_mhash(uint8_t const* s, uint32_t m) {
    uint64_t f = 0, r = 0;
    for (uint32_t i = 0; i < m; ++i) {
        f ^= rol(NT[s[i]], m - 1 - i);
        r ^= rol(NT[3u ^ s[m - 1 - i]], m - 1 - i);
    }
    return f <= r ? f : r;
}

uint32_t best_m(uint32_t k) {
    if (k <= 13) return (k / 2 > k - 4) ? (k / 2) : (k > 4 ? (k - 4) : 1);
    if (k <= 15) return 9;
    if (k <= 21) return 10;
    if (k <= 30) return 11;
    if (k <= 37) return 12;
    if (k <= 42) return 13;
    if (k <= 64) return 14;
    return (k + 2) / 4;
}

// Minimizer value of every (k-1)-mer of a run: mins[j] = min over m-mers
// j .. j+W-1 (W = k - m) of the canonical m-mer hash.  Only the value is used
// downstream, so the reference's tie rule (rightmost) does not change it.
void min_scan(uint8_t const* b, uint32_t L, uint32_t k, uint32_t m, std::vector<uint64_t>& mins) {
    const uint32_t W = k - m;
    const uint32_t nm = L - m + 1;  // m-mers
    std::vector<uint64_t> h(nm);
    for (uint32_t i = 0; i < nm; ++i) h[i] = canon_mhash(b + i, m);
    const uint32_t nk1 = L - (k - 1) + 1;  // (k-1)-mers
    mins.resize(nk1);
    // sliding minimum with a monotone deque (value-only result)
    std::vector<uint32_t> dq(nm);
    size_t head = 0, tail = 0;
    for (uint32_t i = 0; i < nm; ++i) {
        while (tail > head && h[dq[tail - 1]] >= h[i]) --tail;
        dq[tail++] = i;
        if (i + 1 >= W) {
            uint32_t j = i + 1 - W;
            while (dq[head] < j) ++head;
            mins[j] = h[dq[head]];
        }
    }
}

enum : uint8_t { F_BEGIN = 1, F_END = 2, F_OWNS_FIRST = 4, F_OWNS_LAST = 8 };

struct super_occ {
    uint32_t bucket;
    uint8_t flags;
    uint32_t color;
    uint64_t start;  // base offset into the run
    uint32_t len;
};

// Super-k-mers of one ACGT run (bucket_ingester.hpp:36-127).
void emit_supers(uint8_t const* b, uint32_t L, uint32_t k, uint32_t m, uint32_t B, uint32_t color,
                 std::vector<super_occ>& out) {
    const uint32_t K = L - k + 1;
    std::vector<uint64_t> mins;
    min_scan(b, L, k, m, mins);
    auto bucket_of = [&](uint64_t h) { return (uint32_t)((h >> 1) % B); };
    uint32_t run_a = 0;
    bool first_super = true, owns_first = true;
    uint64_t cur = mins[0];
    auto emit = [&](uint32_t fk, uint32_t lk, uint64_t mv, bool beg, bool end, bool of, bool ol) {
        uint8_t f = 0;
        if (beg) f |= F_BEGIN;
        if (end) f |= F_END;
        if (of) f |= F_OWNS_FIRST;
        if (ol) f |= F_OWNS_LAST;
        out.push_back({bucket_of(mv), f, color, fk, lk - fk + k});
    };
    for (uint32_t j = 1; j <= K; ++j) {
        uint64_t nm = mins[j];
        if (nm != cur) {
            uint32_t fk = run_a == 0 ? 0 : run_a - 1;
            emit(fk, j - 1, cur, first_super, false, owns_first, cur < nm);
            first_super = false;
            owns_first = nm < cur;
            cur = nm;
            run_a = j;
        }
    }
    uint32_t fk = run_a == 0 ? 0 : run_a - 1;
    emit(fk, K - 1, cur, first_super, true, owns_first, true);
}

inline uint8_t nuc2(char c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 0xff;
    }
}

// Sequences of a FASTA/FASTQ file (plain or gzip), restating what the
// reference gets from kseq_read (seq_reader.hpp:66): for FASTA the
// concatenation of the lines after a '>' header; for FASTQ the sequence
// line(s) between '@' header and '+'.
std::vector<std::string> read_sequences(std::string const& path) {
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("could not open input file: " + path);
    std::string data;
    char buf[1 << 16];
    int n;
    while ((n = gzread(f, buf, sizeof buf)) > 0) data.append(buf, n);
    gzclose(f);
    std::vector<std::string> seqs;
    size_t p = 0;
    auto next_line = [&](std::string& line) -> bool {
        if (p >= data.size()) return false;
        size_t e = data.find('\n', p);
        if (e == std::string::npos) e = data.size();
        line.assign(data, p, e - p);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        p = e + 1;
        return true;
    };
    std::string line;
    bool have = false;
    // skip to first header
    while (next_line(line))
        if (!line.empty() && (line[0] == '>' || line[0] == '@')) {
            have = true;
            break;
        }
    while (have) {
        bool fastq = line[0] == '@';
        std::string seq;
        have = false;
        while (next_line(line)) {
            if (!line.empty() && (line[0] == '>' || (line[0] == '@' && !fastq))) {
                have = true;
                break;
            }
            if (fastq && !line.empty() && line[0] == '+') {
                // quality: as many characters as the sequence
                size_t q = 0;
                while (q < seq.size() && next_line(line)) q += line.size();
                // next header
                while (next_line(line))
                    if (!line.empty() && (line[0] == '@' || line[0] == '>')) {
                        have = true;
                        break;
                    }
                break;
            }
            seq += line;
        }
        seqs.push_back(std::move(seq));
    }
    return seqs;
}

// ACGT runs of length >= k of a sequence, as 0..3 codes.
void acgt_runs(std::string const& s, uint32_t k, std::vector<std::vector<uint8_t>>& runs) {
    size_t p = 0;
    while (p < s.size()) {
        std::vector<uint8_t> r;
        while (p < s.size()) {
            uint8_t c = nuc2(s[p]);
            if (c == 0xff) break;
            r.push_back(c);
            ++p;
        }
        if (r.size() >= k) runs.push_back(std::move(r));
        while (p < s.size() && nuc2(s[p]) == 0xff) ++p;
    }
}

// ---------------------------------------------------------------- records
void pack2(uint8_t const* src, size_t n, std::vector<uint8_t>& dst) {
    size_t off = dst.size();
    dst.resize(off + (n + 3) / 4, 0);
    for (size_t i = 0; i < n; ++i) dst[off + (i >> 2)] |= (uint8_t)((src[i] & 3u) << (2 * (i & 3)));
}
void varint(uint64_t v, std::vector<uint8_t>& out) {
    while (v >= 0x80) {
        out.push_back((uint8_t)((v & 0x7f) | 0x80));
        v >>= 7;
    }
    out.push_back((uint8_t)v);
}
uint64_t varint_rd(uint8_t const* b, size_t n, size_t& p) {
    uint64_t v = 0;
    unsigned sh = 0;
    while (p < n) {
        uint8_t c = b[p++];
        v |= (uint64_t)(c & 0x7f) << sh;
        if (!(c & 0x80)) return v;
        sh += 7;
        if (sh >= 64) break;
    }
    return v;
}

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// 64-bit key hash of a super-k-mer: splitmix64 finalizer chained over its
// length and its bases taken 32 at a time (base i of a word at bits 2*(i%32),
// missing bases zero).  Shared definition with the GPU phase-1 kernels.
uint64_t super_hash(uint8_t const* b, uint32_t len) {
    uint64_t h = mix64(0x51ed2701f3a5c2b9ULL ^ len);
    for (uint32_t i = 0; i < len; i += 32) {
        uint64_t w = 0;
        uint32_t n = std::min<uint32_t>(32, len - i);
        for (uint32_t j = 0; j < n; ++j) w |= (uint64_t)b[i + j] << (2 * j);
        h = mix64(h ^ w);
    }
    return h;
}

uint32_t bucket_bits(uint32_t B) {
    uint32_t bb = 0;
    while ((1u << bb) < B) ++bb;
    return bb;
}

struct record {
    uint8_t flags;
    std::vector<uint32_t> colors;
    std::vector<uint8_t> bases;
};

// Canonical per-bucket record lists: per bucket, occurrences stably ordered by
// the sort key (bucket << (64-bb)) | (hash >> bb); consecutive occurrences
// with equal key and bases merge (flags AND, colors sorted unique), matching
// the reference compactor's merge rule (bucket_io.hpp:137-166, 229-244).
std::vector<std::vector<record>> canonical_records(
    std::vector<std::vector<uint8_t>> const& bases, std::vector<super_occ> const& occ,
    std::vector<uint32_t> const& occ_run, uint32_t B) {
    const uint32_t bb = bucket_bits(B);
    std::vector<uint64_t> key(occ.size());
    for (size_t i = 0; i < occ.size(); ++i) {
        uint64_t h = super_hash(bases[occ_run[i]].data() + occ[i].start, occ[i].len);
        key[i] = (bb ? ((uint64_t)occ[i].bucket << (64 - bb)) : 0) | (bb ? (h >> bb) : h);
    }
    std::vector<uint32_t> idx(occ.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = (uint32_t)i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    std::vector<std::vector<record>> out(B);
    size_t i = 0;
    while (i < idx.size()) {
        size_t j = i + 1;
        auto const& a = occ[idx[i]];
        uint8_t const* ab = bases[occ_run[idx[i]]].data() + a.start;
        record r;
        r.flags = a.flags;
        r.colors.push_back(a.color);
        while (j < idx.size() && key[idx[j]] == key[idx[i]]) {
            auto const& c = occ[idx[j]];
            uint8_t const* cb = bases[occ_run[idx[j]]].data() + c.start;
            if (c.len != a.len || std::memcmp(ab, cb, a.len) != 0) break;
            r.flags &= c.flags;
            r.colors.push_back(c.color);
            ++j;
        }
        std::sort(r.colors.begin(), r.colors.end());
        r.colors.erase(std::unique(r.colors.begin(), r.colors.end()), r.colors.end());
        r.bases.assign(ab, ab + a.len);
        out[a.bucket].push_back(std::move(r));
        i = j;
    }
    return out;
}

void serialize_record(record const& r, std::vector<uint8_t>& out) {
    varint(r.colors.size(), out);
    uint32_t prev = 0;
    for (uint32_t c : r.colors) {
        varint(c - prev, out);
        prev = c;
    }
    varint(((uint64_t)r.bases.size() << 4) | (r.flags & 0xf), out);
    pack2(r.bases.data(), r.bases.size(), out);
}

std::vector<uint8_t> read_bucket_file(std::string const& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<uint8_t> out, comp;
    for (;;) {
        uint32_t u = 0, c = 0;
        if (std::fread(&u, 4, 1, f) != 1) break;
        if (u == 0) break;
        if (std::fread(&c, 4, 1, f) != 1) {
            std::fclose(f);
            throw std::runtime_error("short read of compressed_size on " + path);
        }
        comp.resize(c);
        if (std::fread(comp.data(), 1, c, f) != c) {
            std::fclose(f);
            throw std::runtime_error("short read of compressed payload on " + path);
        }
        size_t off = out.size();
        out.resize(off + u);
        int d = LZ4_decompress_safe((char const*)comp.data(), (char*)out.data() + off, (int)c, (int)u);
        if (d < 0 || (uint32_t)d != u) {
            std::fclose(f);
            throw std::runtime_error("LZ4_decompress_safe failed on " + path);
        }
    }
    std::fclose(f);
    return out;
}

void write_bucket_file(std::string const& path, std::vector<uint8_t> const& raw) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    if (!raw.empty()) {
        std::vector<char> comp(LZ4_compressBound((int)raw.size()));
        int c = LZ4_compress_default((char const*)raw.data(), comp.data(), (int)raw.size(),
                                     (int)comp.size());
        uint32_t u = (uint32_t)raw.size(), cc = (uint32_t)c;
        std::fwrite(&u, 4, 1, f);
        std::fwrite(&cc, 4, 1, f);
        std::fwrite(comp.data(), 1, c, f);
    }
    uint32_t eof = 0;
    std::fwrite(&eof, 4, 1, f);
    std::fclose(f);
}

// Parse a decompressed bucket stream into records (super_kmer.hpp:121-143).
std::vector<record> parse_records(std::vector<uint8_t> const& buf) {
    std::vector<record> out;
    size_t p = 0;
    while (p < buf.size()) {
        record r;
        uint64_t nc = varint_rd(buf.data(), buf.size(), p);
        uint32_t prev = 0;
        for (uint64_t i = 0; i < nc; ++i) {
            prev += (uint32_t)varint_rd(buf.data(), buf.size(), p);
            r.colors.push_back(prev);
        }
        if (p >= buf.size()) break;
        uint64_t lf = varint_rd(buf.data(), buf.size(), p);
        uint64_t len = lf >> 4;
        r.flags = (uint8_t)(lf & 0xf);
        size_t nb = (len + 3) / 4;
        if (p + nb > buf.size()) break;
        r.bases.resize(len);
        for (uint64_t i = 0; i < len; ++i) r.bases[i] = (buf[p + (i >> 2)] >> (2 * (i & 3))) & 3u;
        p += nb;
        out.push_back(std::move(r));
    }
    return out;
}

// ---------------------------------------------------------------- bits
struct bitbuf {
    std::vector<uint64_t> w;
    uint64_t n = 0;
    void put(uint64_t x, uint32_t len) {
        if (!len) return;
        if (len < 64) x &= (uint64_t(1) << len) - 1;
        uint32_t off = n & 63;
        if (off == 0)
            w.push_back(x);
        else {
            w.back() |= x << off;
            if (off + len > 64) w.push_back(x >> (64 - off));
        }
        n += len;
    }
    void zeros(uint64_t c) {
        while (c >= 64) {
            put(0, 64);
            c -= 64;
        }
        put(0, (uint32_t)c);
    }
};
inline uint32_t msb(uint64_t y) { return 63u - (uint32_t)__builtin_clzll(y); }
void put_gamma(bitbuf& b, uint64_t y) {
    uint32_t l = msb(y);
    b.zeros(l);
    b.put(1, 1);
    b.put(y, l);
}
void put_delta(bitbuf& b, uint64_t x) {
    uint64_t y = x + 1;
    uint32_t l = msb(y);
    put_gamma(b, l + 1);
    b.put(y, l);
}

// hybrid_color_sets.hpp:48-95
void hybrid_encode(bitbuf& b, std::vector<uint32_t> const& s, uint64_t C, uint64_t sparse_t,
                   uint64_t dense_t) {
    put_delta(b, s.size());
    if (s.size() < sparse_t) {
        if (s.empty()) return;
        put_delta(b, s[0]);
        for (size_t i = 1; i < s.size(); ++i) put_delta(b, s[i] - (s[i - 1] + 1));
    } else if (s.size() < dense_t) {
        bitbuf bm;
        bm.zeros(C);
        for (uint32_t c : s) bm.w[c >> 6] |= uint64_t(1) << (c & 63);
        for (uint64_t i = 0; i < C; i += 64) b.put(bm.w[i >> 6], (uint32_t)std::min<uint64_t>(64, C - i));
    } else {
        bool first = true;
        uint32_t prev = 0, val = 0;
        size_t i = 0;
        for (; val < C; ++val) {
            if (i < s.size() && s[i] == val) {
                ++i;
                continue;
            }
            if (first) {
                put_delta(b, val);
                first = false;
            } else
                put_delta(b, val - (prev + 1));
            prev = val;
        }
    }
}

// ---------------------------------------------------------------- phase 2
enum : uint8_t { B_LEFT = 1, B_RIGHT = 2 };
inline bool is_break(uint8_t f) { return f == B_LEFT || f == B_RIGHT; }
static const uint64_t FOREIGN = UINT64_MAX;

struct frag {
    std::string seq;
    std::vector<std::pair<uint64_t, uint32_t>> runs;
    uint8_t open = 0;
};

struct vec_hash {
    size_t operator()(std::vector<uint32_t> const& v) const {
        uint64_t h = 0x12345;
        for (uint32_t x : v) h = mix64(h ^ x);
        return (size_t)h;
    }
};

template <typename K>
struct khash {
    size_t operator()(K x) const {
        return (size_t)(mix64((uint64_t)x) ^ mix64((uint64_t)(x >> 32 >> 32) + 0x9e37));
    }
};

// Global color-set dictionary in first-intern order (streaming_color_set_dict
// semantics, exact equality instead of a 128-bit hash).
struct global_dict {
    uint64_t C, sparse_t, dense_t;
    std::unordered_map<std::vector<uint32_t>, uint64_t, vec_hash> index;
    bitbuf bits;
    std::vector<uint64_t> offsets;
    uint64_t total_integers = 0;
    explicit global_dict(uint64_t c)
        : C(c), sparse_t((uint64_t)(0.25 * c)), dense_t((uint64_t)(0.75 * c)) {}
    uint64_t intern(std::vector<uint32_t> const& s) {
        auto it = index.find(s);
        if (it != index.end()) return it->second;
        uint64_t id = offsets.size();
        offsets.push_back(bits.n);
        hybrid_encode(bits, s, C, sparse_t, dense_t);
        total_integers += s.size();
        index.emplace(s, id);
        return id;
    }
};

template <typename K>
struct bucket_graph {
    uint32_t k;
    struct info {
        K key;
        uint8_t flags = 0;
        bool primary = false;
        std::vector<uint32_t> rsids;  // owned contributions
        uint32_t cid = UINT32_MAX;
    };
    std::vector<info> nodes;                    // insertion order
    std::unordered_map<K, uint32_t, khash<K>> at;  // key -> node index

    info* find(K x) {
        auto it = at.find(x);
        return it == at.end() ? nullptr : &nodes[it->second];
    }
    uint32_t index_of(K x) const { return at.find(x)->second; }

    uint8_t ext_mask(K can) {
        uint8_t out = 0;
        const K msk = kmask<K>(k);
        K fwd = can, rev = revcomp(can, k);
        for (uint32_t nt = 0; nt < 4; ++nt) {
            if (find(canon(((fwd << 2) | nt) & msk, k))) out |= (uint8_t)(1u << nt);
            if (find(canon(((rev << 2) | nt) & msk, k))) out |= (uint8_t)(1u << (4 + nt));
        }
        return out;
    }
    static uint8_t fnib(uint8_t m, bool rc) { return (uint8_t)((rc ? (m >> 4) : m) & 0xf); }
    static uint8_t bnib(uint8_t m, bool rc) { return (uint8_t)((rc ? m : (m >> 4)) & 0xf); }
    void bstep(K can, bool rc, uint32_t nt, K& nc, bool& nrc) {
        K cur = rc ? revcomp(can, k) : can;
        K nf = ((cur << 2) | nt) & kmask<K>(k);
        K nr = revcomp(nf, k);
        if (nf <= nr) {
            nc = nf;
            nrc = false;
        } else {
            nc = nr;
            nrc = true;
        }
    }
    bool walk_step(K can, bool rc, bool forward, K& nc, bool& nrc) {
        uint8_t m = ext_mask(can);
        uint8_t nib = forward ? fnib(m, rc) : bnib(m, rc);
        if (__builtin_popcount(nib) != 1) return false;
        uint32_t nt = (uint32_t)__builtin_ctz(nib);
        if (forward)
            bstep(can, rc, nt, nc, nrc);
        else {
            bstep(can, !rc, nt, nc, nrc);
            nrc = !nrc;
        }
        uint8_t nm = ext_mask(nc);
        uint8_t facing = forward ? bnib(nm, nrc) : fnib(nm, nrc);
        return __builtin_popcount(facing) == 1;
    }
};

template <typename K>
std::string kstr(K x, uint32_t k) {
    std::string s(k, 'N');
    for (uint32_t i = 0; i < k; ++i) {
        s[k - 1 - i] = "ACGT"[(uint32_t)(x & 3)];
        x >>= 2;
    }
    return s;
}

// process_bucket (bucket_walker.hpp:338-570) for one bucket's records, then
// the merge of its local classes into `gd` (bucket_walker.hpp:713-757).
template <typename K>
void process_bucket(std::vector<record> const& recs, uint32_t k, global_dict& gd,
                    std::vector<frag>& frags) {
    bucket_graph<K> g;
    g.k = k;
    const K msk = kmask<K>(k);
    // record-set dictionary: distinct color lists -> rsid (first-intern order)
    std::unordered_map<std::vector<uint32_t>, uint32_t, vec_hash> rs_index;
    std::vector<std::vector<uint32_t>> rs_lists;
    for (auto const& r : recs) {
        if (r.bases.size() < k) continue;
        uint32_t rsid;
        auto it = rs_index.find(r.colors);
        if (it == rs_index.end()) {
            rsid = (uint32_t)rs_lists.size();
            rs_lists.push_back(r.colors);
            rs_index.emplace(r.colors, rsid);
        } else
            rsid = it->second;
        const bool begin_incl = r.flags & F_BEGIN, end_incl = r.flags & F_END;
        const bool of = r.flags & F_OWNS_FIRST, ol = r.flags & F_OWNS_LAST;
        const uint32_t nk = (uint32_t)(r.bases.size() - (k - 1));
        K fwd = 0, rc = 0;
        for (uint32_t i = 0; i < k - 1; ++i) {
            fwd = ((fwd << 2) | r.bases[i]) & msk;
            rc = (rc >> 2) | ((K)(r.bases[i] ^ 3) << (2 * (k - 1)));
        }
        for (uint32_t idx = 0; idx < nk; ++idx) {
            uint8_t v = r.bases[idx + k - 1];
            fwd = ((fwd << 2) | v) & msk;
            rc = (rc >> 2) | ((K)(v ^ 3) << (2 * (k - 1)));
            bool isf = fwd <= rc;
            K can = isf ? fwd : rc;
            uint8_t contrib = 0;
            if (!begin_incl && idx == 0) contrib |= isf ? B_LEFT : B_RIGHT;
            if (!end_incl && idx == nk - 1) contrib |= isf ? B_RIGHT : B_LEFT;
            auto ins = g.at.emplace(can, (uint32_t)g.nodes.size());
            if (ins.second) {
                g.nodes.emplace_back();
                g.nodes.back().key = can;
            }
            auto& inf = g.nodes[ins.first->second];
            inf.flags |= contrib;
            bool owned = !((idx == 0 && !of) || (idx == nk - 1 && !ol));
            if (owned) {
                inf.rsids.push_back(rsid);
                inf.primary = true;
            }
        }
    }
    // resolve: local classes in first-appearance order
    std::unordered_map<std::vector<uint32_t>, uint32_t, vec_hash> local_index;
    std::vector<std::vector<uint32_t>> local_lists;
    for (auto& n : g.nodes) {
        if (!n.primary) continue;
        std::vector<uint32_t> rs = n.rsids;
        std::sort(rs.begin(), rs.end());
        rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
        std::vector<uint32_t> set;
        for (uint32_t r : rs) set.insert(set.end(), rs_lists[r].begin(), rs_lists[r].end());
        std::sort(set.begin(), set.end());
        set.erase(std::unique(set.begin(), set.end()), set.end());
        auto it = local_index.find(set);
        if (it == local_index.end()) {
            n.cid = (uint32_t)local_lists.size();
            local_index.emplace(set, n.cid);
            local_lists.push_back(std::move(set));
        } else
            n.cid = it->second;
    }
    // walk (bucket_walker.hpp:431-566)
    std::vector<uint8_t> visited(g.nodes.size(), 0);
    std::vector<frag> local;
    auto push = [](frag& u, uint64_t c) {
        if (!u.runs.empty() && u.runs.back().first == c)
            u.runs.back().second += 1;
        else
            u.runs.push_back({c, 1});
    };
    for (uint32_t si = 0; si < g.nodes.size(); ++si) {
        if (visited[si]) continue;
        const K seed = g.nodes[si].key;
        visited[si] = 1;
        const uint8_t sf = g.nodes[si].flags;
        std::vector<std::pair<K, bool>> bw, fw;
        bool ol = false, orr = false;
        auto ldeg_back = [&](K c, bool rc) {
            return __builtin_popcount(bucket_graph<K>::bnib(g.ext_mask(c), rc));
        };
        auto ldeg_fwd = [&](K c, bool rc) {
            return __builtin_popcount(bucket_graph<K>::fnib(g.ext_mask(c), rc));
        };
        for (int dir = 0; dir < 2; ++dir) {
            const bool forward = dir == 1;
            if (!forward && sf == B_LEFT) {
                ol = ldeg_back(seed, false) <= 1;
                continue;
            }
            if (forward && sf == B_RIGHT) {
                orr = ldeg_fwd(seed, false) <= 1;
                continue;
            }
            K c = seed;
            bool rc = false;
            for (;;) {
                K nc;
                bool nrc;
                if (!g.walk_step(c, rc, forward, nc, nrc)) break;
                uint32_t ni = g.index_of(nc);
                if (visited[ni]) break;
                visited[ni] = 1;
                (forward ? fw : bw).push_back({nc, nrc});
                c = nc;
                rc = nrc;
                if (is_break(g.nodes[ni].flags)) {
                    if (forward)
                        orr = ldeg_fwd(c, rc) <= 1;
                    else
                        ol = ldeg_back(c, rc) <= 1;
                    break;
                }
            }
        }
        frag u;
        bool first = true;
        auto app = [&](std::pair<K, bool> const& p) {
            K w = p.second ? revcomp(p.first, k) : p.first;
            if (first) {
                u.seq = kstr(w, k);
                first = false;
            } else
                u.seq.push_back("ACGT"[(uint32_t)(w & 3)]);
            auto const& inf = g.nodes[g.index_of(p.first)];
            push(u, inf.primary ? (uint64_t)inf.cid : FOREIGN);
        };
        for (auto it = bw.rbegin(); it != bw.rend(); ++it) app(*it);
        app({seed, false});
        for (auto const& p : fw) app(p);
        if (ol) u.open |= 1;
        if (orr) u.open |= 2;
        local.push_back(std::move(u));
    }
    // merge local classes into the global dict, in local order
    std::vector<uint64_t> l2g(local_lists.size());
    for (size_t i = 0; i < local_lists.size(); ++i) l2g[i] = gd.intern(local_lists[i]);
    for (auto& u : local)
        for (auto& r : u.runs)
            if (r.first != FOREIGN) r.first = l2g[r.first];
    for (auto& u : local) frags.push_back(std::move(u));
}

void append_frag(frag const& u, std::vector<uint8_t>& out) {
    auto put = [&](void const* p, size_t n) {
        out.insert(out.end(), (uint8_t const*)p, (uint8_t const*)p + n);
    };
    uint32_t nr = (uint32_t)u.runs.size(), sl = (uint32_t)u.seq.size();
    put(&u.open, 1);
    put(&nr, 4);
    for (auto const& r : u.runs) {
        put(&r.first, 8);
        put(&r.second, 4);
    }
    put(&sl, 4);
    put(u.seq.data(), sl);
}

// Finalized .color_sets layout (streaming_color_set_dict.hpp:221-294) with the
// Elias-Fano offsets serialized in the stand-in `bits` layout of oracle/shim.
void write_color_sets(global_dict const& gd, std::string const& path) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open " + path);
    uint32_t C = (uint32_t)gd.C, st = (uint32_t)gd.sparse_t, dt = (uint32_t)gd.dense_t;
    uint64_t nbits = gd.bits.n, nwords = (nbits + 63) / 64;
    std::fwrite(&C, 4, 1, f);
    std::fwrite(&st, 4, 1, f);
    std::fwrite(&dt, 4, 1, f);
    std::fwrite(&nbits, 8, 1, f);
    std::fwrite(&nwords, 8, 1, f);
    if (nwords) std::fwrite(gd.bits.w.data(), 8, nwords, f);
    // Elias-Fano over offsets + sentinel
    std::vector<uint64_t> v = gd.offsets;
    v.push_back(nbits);
    uint64_t n = v.size(), U = nbits, l = 0;
    if (n > 0 && U > n) {
        uint64_t q = U / n;
        while ((uint64_t(1) << (l + 1)) <= q) ++l;
    }
    bitbuf low, high;
    high.zeros(n + (U >> l) + 1);
    for (uint64_t i = 0; i < n; ++i) {
        if (l) low.put(v[i], (uint32_t)l);
        uint64_t p = (v[i] >> l) + i;
        high.w[p >> 6] |= uint64_t(1) << (p & 63);
    }
    auto wbv = [&](bitbuf const& b) {
        uint64_t nb = b.n, sz = b.w.size();
        std::fwrite(&nb, 8, 1, f);
        std::fwrite(&sz, 8, 1, f);
        if (sz) std::fwrite(b.w.data(), 8, sz, f);
    };
    std::fwrite(&U, 8, 1, f);
    std::fwrite(&n, 8, 1, f);
    std::fwrite(&l, 8, 1, f);
    wbv(low);
    wbv(high);
    std::fclose(f);
}

thread_local std::string g_err;

}  // namespace oracle

using namespace oracle;

static std::vector<std::string> read_list(char const* p) {
    std::vector<std::string> files;
    std::ifstream in(p);
    std::string line;
    while (std::getline(in, line))
        if (!line.empty()) files.push_back(line);
    return files;
}

extern "C" {

char const* oracle_last_error() { return g_err.c_str(); }

uint32_t oracle_best_m(uint32_t k) { return best_m(k); }

// Canonical ntHash of every m-mer of a 0..3 base array.
void oracle_mhashes(uint8_t const* b, uint32_t L, uint32_t m, uint64_t* out) {
    for (uint32_t i = 0; i + m <= L; ++i) out[i] = canon_mhash(b + i, m);
}

// Minimizer value of every (k-1)-mer of a run (L - k + 2 values).
void oracle_kminus1_minimizers(uint8_t const* b, uint32_t L, uint32_t k, uint32_t m, uint64_t* out) {
    std::vector<uint64_t> mins;
    min_scan(b, L, k, m, mins);
    std::memcpy(out, mins.data(), mins.size() * 8);
}

uint64_t oracle_super_hash(uint8_t const* b, uint32_t len) { return super_hash(b, len); }

// Phase 1 over a filenames list: dumps every super-k-mer occurrence in the
// layout of oracle/ref_harness/ref_phase1.cpp; when bucket_dir is non-null also
// writes canonical bucket files bucket_<b>.bin (one LZ4 frame each).
int oracle_phase1_from(char const* filelist, uint32_t first_color, uint32_t k, uint32_t m, uint32_t B,
                       char const* dump_path, char const* bucket_dir, uint64_t* n_supers, uint64_t* n_kmers);

int oracle_phase1(char const* filelist, uint32_t k, uint32_t m, uint32_t B, char const* dump_path,
                  char const* bucket_dir, uint64_t* n_supers, uint64_t* n_kmers) {
    return oracle_phase1_from(filelist, 0, k, m, B, dump_path, bucket_dir, n_supers, n_kmers);
}

// Phase 1 with file i of the list read as color first_color + i (one rank's
// slice of a collection split by input file).
int oracle_phase1_from(char const* filelist, uint32_t first_color, uint32_t k, uint32_t m, uint32_t B,
                       char const* dump_path, char const* bucket_dir, uint64_t* n_supers, uint64_t* n_kmers) {
    try {
        if (m == 0) m = best_m(k);
        auto files = read_list(filelist);
        std::vector<std::vector<uint8_t>> runs;
        std::vector<super_occ> occ;
        std::vector<uint32_t> occ_run;
        uint64_t nk = 0;
        for (uint32_t c = 0; c < files.size(); ++c) {
            for (auto const& s : read_sequences(files[c])) {
                size_t r0 = runs.size();
                acgt_runs(s, k, runs);
                for (size_t r = r0; r < runs.size(); ++r) {
                    size_t o0 = occ.size();
                    nk += runs[r].size() - k + 1;
                    emit_supers(runs[r].data(), (uint32_t)runs[r].size(), k, m, B, first_color + c, occ);
                    for (size_t o = o0; o < occ.size(); ++o) occ_run.push_back((uint32_t)r);
                }
            }
        }
        if (n_supers) *n_supers = occ.size();
        if (n_kmers) *n_kmers = nk;
        if (dump_path) {
            std::FILE* f = std::fopen(dump_path, "wb");
            if (!f) throw std::runtime_error("cannot open dump");
            uint64_t n = occ.size();
            std::fwrite(&n, 8, 1, f);
            std::vector<uint8_t> pk;
            for (size_t i = 0; i < occ.size(); ++i) {
                auto const& o = occ[i];
                std::fwrite(&o.bucket, 4, 1, f);
                std::fwrite(&o.flags, 1, 1, f);
                std::fwrite(&o.color, 4, 1, f);
                std::fwrite(&o.len, 4, 1, f);
                pk.clear();
                pack2(runs[occ_run[i]].data() + o.start, o.len, pk);
                std::fwrite(pk.data(), 1, pk.size(), f);
            }
            std::fclose(f);
        }
        if (bucket_dir) {
            auto recs = canonical_records(runs, occ, occ_run, B);
            for (uint32_t b = 0; b < B; ++b) {
                std::vector<uint8_t> raw;
                for (auto const& r : recs[b]) serialize_record(r, raw);
                write_bucket_file(std::string(bucket_dir) + "/bucket_" + std::to_string(b) + ".bin", raw);
            }
        }
        return 0;
    } catch (std::exception const& e) {
        g_err = e.what();
        return -1;
    }
}

// k-mer occurrences per bucket (the super-k-mers' k-mers, before any
// deduplication) of a filenames list: counts[B].  Test aid: shows how skewed
// a workload's buckets are.
int oracle_bucket_kmers(char const* filelist, uint32_t k, uint32_t m, uint32_t B, uint64_t* counts) {
    try {
        if (m == 0) m = best_m(k);
        auto files = read_list(filelist);
        for (uint32_t b = 0; b < B; ++b) counts[b] = 0;
        std::vector<std::vector<uint8_t>> runs;
        std::vector<super_occ> occ;
        for (uint32_t c = 0; c < files.size(); ++c) {
            for (auto const& s : read_sequences(files[c])) {
                runs.clear();
                acgt_runs(s, k, runs);
                for (auto const& r : runs) {
                    occ.clear();
                    emit_supers(r.data(), (uint32_t)r.size(), k, m, B, c, occ);
                    for (auto const& o : occ) counts[o.bucket] += o.len - k + 1;
                }
            }
        }
        return 0;
    } catch (std::exception const& e) {
        g_err = e.what();
        return -1;
    }
}

// Phase 2 over a directory of bucket files, buckets 0..B-1 in order (the
// reference's process_buckets at one thread): writes <out_dir>/frag_unitigs.bin
// and <out_dir>/out.color_sets (finalized).
int oracle_phase2(char const* bucket_dir, uint32_t B, uint32_t k, uint32_t C, char const* out_dir,
                  uint64_t* n_frags, uint64_t* n_color_sets, uint64_t* total_seq) {
    try {
        global_dict gd(C);
        std::vector<frag> frags;
        for (uint32_t b = 0; b < B; ++b) {
            std::string p = std::string(bucket_dir) + "/bucket_" + std::to_string(b) + ".bin";
            std::FILE* t = std::fopen(p.c_str(), "rb");
            if (!t) continue;
            std::fclose(t);
            auto recs = parse_records(read_bucket_file(p));
            if (k <= 31)
                process_bucket<uint64_t>(recs, k, gd, frags);
            else
                process_bucket<u128>(recs, k, gd, frags);
        }
        std::vector<uint8_t> out;
        uint64_t ts = 0;
        for (auto const& u : frags) {
            append_frag(u, out);
            ts += u.seq.size();
        }
        std::string fp = std::string(out_dir) + "/frag_unitigs.bin";
        std::FILE* f = std::fopen(fp.c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open " + fp);
        if (!out.empty()) std::fwrite(out.data(), 1, out.size(), f);
        std::fclose(f);
        write_color_sets(gd, std::string(out_dir) + "/out.color_sets");
        if (n_frags) *n_frags = frags.size();
        if (n_color_sets) *n_color_sets = gd.offsets.size();
        if (total_seq) *total_seq = ts;
        return 0;
    } catch (std::exception const& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
