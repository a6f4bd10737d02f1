// Seeded synthetic pangenome generator for the benchmark and test workloads.
//
// A collection is a set of genomes (one color each) derived from one seeded
// uniform-ACGT ancestor:
//   * optional low-complexity content in the ancestor (homopolymer runs and
//     dinucleotide repeats of 10-100 bp) up to `lowcomp_frac` of its length;
//   * optional tandem-repeat arrays in the ancestor (unit period 2-200 bp,
//     5-50 copies) up to `tandem_frac` of its length;
//   * per genome: a window of the ancestor (length log-uniform in
//     [len_min, len_max], the whole ancestor when they are equal), SNPs at a
//     rate drawn uniformly in [div_min, div_max], `indels` indels of 1-50 bp,
//     one insertion drawn from a pool of `mobile_pool` random elements of
//     mobile_min..mobile_max bp, `repeats_per_genome` insertions drawn from a
//     pool of `repeat_pool` shared 1-5 kbp repeats, then a split into
//     contigs_min..contigs_max contigs (log-uniform when contigs_log is set).
// Every random choice comes from a splitmix64 stream seeded by (seed, genome
// index), so any genome can be regenerated alone and in parallel.
//
// C entry points (see include/cdbg_synth.h): generate one genome into a
// caller buffer, or write a whole collection as FASTA (optionally gzipped)
// plus a filenames list (line i = color i), the input format of the
// reference's cdbg-build -i.

#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "cdbg_synth.h"

namespace {

struct rng {
    uint64_t s;
    explicit rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    // uniform integer in [a, b]
    uint64_t range(uint64_t a, uint64_t b) {
        return a + (uint64_t)(((__uint128_t)next() * (b - a + 1)) >> 64);
    }
    double uniform(double a, double b) { return a + (b - a) * unit(); }
    double log_uniform(double a, double b) {
        if (a == b) return a;
        return std::exp(uniform(std::log(a), std::log(b)));
    }
    char base() { return "ACGT"[next() >> 62]; }
};

uint64_t mix_seed(uint64_t seed, uint64_t a, uint64_t b) {
    rng r(seed ^ (a * 0xd1b54a32d192ed03ULL) ^ (b * 0x8cb92ba72f3d8dd7ULL));
    r.next();
    return r.next();
}

std::string random_seq(rng& r, uint64_t n) {
    std::string s(n, 'A');
    for (uint64_t i = 0; i < n; ++i) s[i] = r.base();
    return s;
}

// Overwrite stretches of `s` with structured content until `frac` of it is
// covered. kind 0 = low complexity (homopolymers / dinucleotides 10-100 bp),
// kind 1 = tandem repeats (period 2-200, 5-50 copies).
void add_structured(std::string& s, double frac, int kind, rng& r) {
    if (frac <= 0 || s.empty()) return;
    const uint64_t target = (uint64_t)(frac * (double)s.size());
    uint64_t covered = 0;
    while (covered < target) {
        std::string piece;
        if (kind == 0) {
            uint64_t len = r.range(10, 100);
            if (r.next() & 1) {
                piece.assign(len, r.base());
            } else {
                char a = r.base(), b = r.base();
                while (b == a) b = r.base();
                piece.resize(len);
                for (uint64_t i = 0; i < len; ++i) piece[i] = (i & 1) ? b : a;
            }
        } else {
            uint64_t period = r.range(2, 200), copies = r.range(5, 50);
            std::string unit = random_seq(r, period);
            for (uint64_t c = 0; c < copies; ++c) piece += unit;
        }
        if (piece.size() >= s.size()) piece.resize(s.size() / 2);
        uint64_t pos = r.range(0, s.size() - piece.size());
        std::memcpy(&s[pos], piece.data(), piece.size());
        covered += piece.size();
    }
}

struct collection {
    cdbg_synth_params p;
    std::string ancestor;
    std::vector<std::string> mobiles;
    std::vector<std::string> repeats;

    explicit collection(cdbg_synth_params const& params) : p(params) {
        rng r(mix_seed(p.seed, 0xA11CE, 0));
        const uint64_t alen = (uint64_t)std::max(p.len_max, p.len_min);
        ancestor = random_seq(r, alen);
        add_structured(ancestor, p.lowcomp_frac, 0, r);
        add_structured(ancestor, p.tandem_frac, 1, r);
        for (uint32_t i = 0; i < p.mobile_pool; ++i)
            mobiles.push_back(random_seq(r, r.range(p.mobile_min, std::max(p.mobile_min, p.mobile_max))));
        for (uint32_t i = 0; i < p.repeat_pool; ++i)
            repeats.push_back(random_seq(r, r.range(1000, 5000)));
    }

    // Genome g as a list of contigs.
    std::vector<std::string> genome(uint32_t g) const {
        rng r(mix_seed(p.seed, 0x6E0, g + 1));
        const uint64_t alen = ancestor.size();
        uint64_t len = (uint64_t)r.log_uniform(p.len_min, p.len_max);
        len = std::min<uint64_t>(std::max<uint64_t>(len, 1000), alen);
        uint64_t start = (len < alen) ? r.range(0, alen - len) : 0;
        std::string s = ancestor.substr(start, len);
        // SNPs by geometric gaps at rate d.
        const double d = r.uniform(p.div_min, p.div_max);
        if (d > 0) {
            const double lq = std::log1p(-d);
            uint64_t pos = 0;
            for (;;) {
                double u = r.unit();
                uint64_t gap = (uint64_t)std::floor(std::log1p(-u) / lq);
                pos += gap;
                if (pos >= s.size()) break;
                char c = s[pos], b = r.base();
                while (b == c) b = r.base();
                s[pos] = b;
                ++pos;
            }
        }
        for (uint32_t i = 0; i < p.indels && s.size() > 100; ++i) {
            uint64_t l = r.range(1, 50);
            uint64_t pos = r.range(0, s.size() - 60);
            if (r.next() & 1)
                s.insert(pos, random_seq(r, l));
            else
                s.erase(pos, l);
        }
        if (!mobiles.empty()) {
            std::string const& m = mobiles[r.range(0, mobiles.size() - 1)];
            s.insert(r.range(0, s.size()), m);
        }
        if (!repeats.empty()) {
            for (uint32_t i = 0; i < p.repeats_per_genome; ++i) {
                std::string const& m = repeats[r.range(0, repeats.size() - 1)];
                s.insert(r.range(0, s.size()), m);
            }
        }
        uint32_t nc = p.contigs_log
                          ? (uint32_t)std::floor(r.log_uniform(p.contigs_min, p.contigs_max + 0.999))
                          : (uint32_t)r.range(p.contigs_min, p.contigs_max);
        nc = std::max<uint32_t>(1, std::min<uint32_t>(nc, (uint32_t)(s.size() / 100 + 1)));
        std::vector<uint64_t> cuts;
        for (uint32_t i = 1; i < nc; ++i) cuts.push_back(r.range(1, s.size() - 1));
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
        std::vector<std::string> out;
        uint64_t prev = 0;
        for (uint64_t c : cuts) {
            out.push_back(s.substr(prev, c - prev));
            prev = c;
        }
        out.push_back(s.substr(prev));
        // Lower-case a short stretch now and then so parsers see both cases.
        if (p.lowercase_runs) {
            for (auto& c : out)
                if (c.size() > 200 && (r.next() & 3) == 0) {
                    uint64_t a = r.range(0, c.size() - 100);
                    for (uint64_t i = a; i < a + 50; ++i) c[i] = (char)(c[i] | 0x20);
                }
        }
        if (p.n_runs) {
            for (auto& c : out)
                if (c.size() > 400 && (r.next() & 3) == 0) {
                    uint64_t a = r.range(100, c.size() - 200);
                    uint64_t l = r.range(1, 60);
                    for (uint64_t i = a; i < a + l; ++i) c[i] = 'N';
                }
        }
        return out;
    }
};

}  // namespace

extern "C" {

int64_t cdbg_synth_genome(cdbg_synth_params const* params, uint32_t g, char* out, uint64_t cap,
                          uint64_t* contig_lens, uint32_t contig_cap, uint32_t* num_contigs) {
    try {
        collection c(*params);
        auto contigs = c.genome(g);
        uint64_t total = 0;
        for (auto const& s : contigs) total += s.size();
        if (num_contigs) *num_contigs = (uint32_t)contigs.size();
        if (out == nullptr) return (int64_t)total;
        if (total > cap || contigs.size() > contig_cap) return -1;
        uint64_t off = 0;
        for (size_t i = 0; i < contigs.size(); ++i) {
            std::memcpy(out + off, contigs[i].data(), contigs[i].size());
            off += contigs[i].size();
            if (contig_lens) contig_lens[i] = contigs[i].size();
        }
        return (int64_t)total;
    } catch (...) {
        return -2;
    }
}

// Generate genomes [g0, g1) into one caller buffer, back to back, with
// per-contig lengths and the number of contigs per genome. Threads generate
// disjoint genomes; the caller sizes `out` by a first call with out == NULL,
// which returns the total byte count and the total contig count.
int64_t cdbg_synth_collection(cdbg_synth_params const* params, uint32_t g0, uint32_t g1,
                              uint32_t threads, char* out, uint64_t cap, uint64_t* contig_lens,
                              uint64_t contig_cap, uint32_t* contigs_per_genome,
                              uint64_t* total_contigs) {
    try {
        collection c(*params);
        const uint32_t n = g1 > g0 ? g1 - g0 : 0;
        std::vector<std::vector<std::string>> gen(n);
        if (threads == 0) threads = 1;
        std::atomic<uint32_t> next{0};
        std::vector<std::thread> ts;
        for (uint32_t t = 0; t < threads; ++t)
            ts.emplace_back([&] {
                for (;;) {
                    uint32_t i = next.fetch_add(1);
                    if (i >= n) break;
                    gen[i] = c.genome(g0 + i);
                }
            });
        for (auto& t : ts) t.join();
        uint64_t bytes = 0, ncont = 0;
        for (auto const& g : gen) {
            ncont += g.size();
            for (auto const& s : g) bytes += s.size();
        }
        if (total_contigs) *total_contigs = ncont;
        if (out == nullptr) return (int64_t)bytes;
        if (bytes > cap || ncont > contig_cap) return -1;
        uint64_t off = 0, ci = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (contigs_per_genome) contigs_per_genome[i] = (uint32_t)gen[i].size();
            for (auto const& s : gen[i]) {
                std::memcpy(out + off, s.data(), s.size());
                off += s.size();
                if (contig_lens) contig_lens[ci] = s.size();
                ++ci;
            }
        }
        return (int64_t)bytes;
    } catch (...) {
        return -2;
    }
}

int cdbg_synth_write_fasta(cdbg_synth_params const* params, uint32_t g0, uint32_t g1,
                           char const* out_dir, int gzip_level, uint32_t threads,
                           char const* filelist_path) {
    try {
        collection c(*params);
        const uint32_t n = g1 > g0 ? g1 - g0 : 0;
        std::vector<std::string> paths(n);
        for (uint32_t i = 0; i < n; ++i)
            paths[i] = std::string(out_dir) + "/g" + std::to_string(g0 + i) +
                       (gzip_level > 0 ? ".fa.gz" : ".fa");
        if (threads == 0) threads = 1;
        std::atomic<uint32_t> next{0};
        std::atomic<int> err{0};
        std::vector<std::thread> ts;
        for (uint32_t t = 0; t < threads; ++t)
            ts.emplace_back([&] {
                std::string buf;
                for (;;) {
                    uint32_t i = next.fetch_add(1);
                    if (i >= n) break;
                    auto contigs = c.genome(g0 + i);
                    buf.clear();
                    for (size_t ci = 0; ci < contigs.size(); ++ci) {
                        buf += ">g" + std::to_string(g0 + i) + "_c" + std::to_string(ci) + "\n";
                        auto const& s = contigs[ci];
                        for (size_t p = 0; p < s.size(); p += 80) {
                            buf.append(s, p, std::min<size_t>(80, s.size() - p));
                            buf += '\n';
                        }
                    }
                    if (gzip_level > 0) {
                        char mode[16];
                        std::snprintf(mode, sizeof mode, "wb%d", gzip_level > 9 ? 9 : gzip_level);
                        gzFile f = gzopen(paths[i].c_str(), mode);
                        if (!f || gzwrite(f, buf.data(), (unsigned)buf.size()) != (int)buf.size()) {
                            err = 1;
                            if (f) gzclose(f);
                            continue;
                        }
                        gzclose(f);
                    } else {
                        std::FILE* f = std::fopen(paths[i].c_str(), "wb");
                        if (!f || std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) err = 1;
                        if (f) std::fclose(f);
                    }
                }
            });
        for (auto& t : ts) t.join();
        if (err) return -1;
        std::FILE* lf = std::fopen(filelist_path, "w");
        if (!lf) return -1;
        for (auto const& p : paths) std::fprintf(lf, "%s\n", p.c_str());
        std::fclose(lf);
        return 0;
    } catch (...) {
        return -2;
    }
}

}  // extern "C"
