// Host-side I/O for the GPU phases (see io.hpp).

#include "io.hpp"

#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <stdexcept>
#include <thread>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/vfs.h>
#include <unistd.h>

extern "C" {
// System LZ4 block API (liblz4.so.1), the functions the reference calls at
// bucket_io.hpp:259-263 and :695.
int LZ4_compressBound(int inputSize);
int LZ4_compress_default(const char* src, char* dst, int srcSize, int dstCapacity);
int LZ4_decompress_safe(const char* src, char* dst, int compressedSize, int dstCapacity);
}
// LZ4's largest block input (lz4.h LZ4_MAX_INPUT_SIZE)
static constexpr uint64_t LZ4_MAX_INPUT = 0x7E000000;

namespace cdbg {
namespace io {

namespace {
inline bool is_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// A compression output buffer per thread, kept between frames (a fresh
// multi-MB buffer per frame costs its page faults every time).
std::vector<char>& lz4_scratch(size_t n) {
    thread_local std::vector<char> buf;
    if (buf.size() < n) buf.resize(n);
    return buf;
}

template <typename F>
void parallel_for(size_t n, uint32_t threads, F&& f) {
    if (threads <= 1 || n <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> ts;
    std::exception_ptr err;
    std::atomic<bool> failed{false};
    for (uint32_t t = 0; t < threads && t < n; ++t)
        ts.emplace_back([&] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n || failed) break;
                try {
                    f(i);
                } catch (...) {
                    if (!failed.exchange(true)) err = std::current_exception();
                }
            }
        });
    for (auto& t : ts) t.join();
    if (err) std::rethrow_exception(err);
}
}  // namespace

bool parse_fastx(char const* d, size_t n, std::function<void(char const*, size_t)> const& emit) {
    size_t p = 0;
    int last = 0;
    std::string seq;
    for (;;) {
        if (last == 0) {
            while (p < n && d[p] != '>' && d[p] != '@') ++p;
            if (p >= n) return true;
            last = d[p++];
        }
        // name up to whitespace; the rest of the header line is a comment
        if (p >= n) return true;  // header char at EOF: nothing to read
        char c = 0;
        while (p < n && !is_space(d[p])) ++p;
        if (p < n) c = d[p++];
        if (c != '\n')
            while (p < n && d[p++] != '\n') {
            }
        seq.clear();
        int cc = -1;
        while (p < n) {
            cc = (unsigned char)d[p++];
            if (cc == '>' || cc == '+' || cc == '@') break;
            cc = -1;
            if (d[p - 1] == '\n') continue;
            size_t e = p - 1;
            while (p < n && d[p] != '\n') ++p;
            seq.append(d + e, p - e);
            if (p < n) ++p;  // newline
        }
        if (cc == '>' || cc == '@') last = cc;
        if (cc != '+') {
            emit(seq.data(), seq.size());
            if (cc == -1) return true;
            continue;
        }
        // FASTQ quality: skip the '+' line, then read seq.size() printable chars
        while (p < n && d[p] != '\n') ++p;
        if (p >= n) return false;
        ++p;
        size_t q = 0;
        while (p < n) {
            unsigned char qc = (unsigned char)d[p++];
            if (q >= seq.size()) break;
            if (qc >= 33 && qc <= 127) ++q;
        }
        last = 0;
        if (q != seq.size()) return false;
        emit(seq.data(), seq.size());
    }
}

std::string slurp(std::string const& path) {
    // inflate straight into a buffer sized from the file's size hint (grown
    // if the file inflates to more), no intermediate copy
    const uint64_t hint = inflated_size_hint(path);
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("could not open input file: " + path);
    gzbuffer(f, 1 << 18);
    std::string out;
    out.resize((size_t)std::max<uint64_t>(hint, 4096) + 1);
    size_t n = 0;
    for (;;) {
        if (n == out.size()) out.resize(out.size() * 2);
        const size_t want = std::min<size_t>(out.size() - n, 1u << 30);
        const int r = gzread(f, &out[n], (unsigned)want);
        if (r < 0) {
            gzclose(f);
            throw std::runtime_error("gzip read error on " + path);
        }
        if (r == 0) break;
        n += (size_t)r;
    }
    gzclose(f);
    out.resize(n);
    return out;
}

namespace {
// FASTA records of d[0, n) with the same rules as parse_fastx, the sequence
// bytes appended to `seq` and one length per record to `lens`, scanning lines
// with memchr.  Returns false, with seq and lens left as they were, on a
// header or line start that parse_fastx reads as FASTQ ('@' header or a '+'
// line): the caller then parses the file with parse_fastx.
bool parse_fasta_fast(char const* d, size_t n, std::string& seq, std::vector<uint64_t>& lens) {
    const size_t seq0 = seq.size(), lens0 = lens.size();
    auto fail = [&] {
        seq.resize(seq0);
        lens.resize(lens0);
        return false;
    };
    size_t p = 0;
    int last = 0;
    for (;;) {
        if (last == 0) {
            while (p < n && d[p] != '>' && d[p] != '@') ++p;
            if (p >= n) return true;
            last = d[p++];
        }
        if (last == '@') return fail();
        if (p >= n) return true;  // header char at EOF: nothing to read
        char c = 0;
        while (p < n && !is_space(d[p])) ++p;
        if (p < n) c = d[p++];
        if (c != '\n') {
            void const* q = std::memchr(d + p, '\n', n - p);
            p = q ? (size_t)((char const*)q - d) + 1 : n;
        }
        const size_t start = seq.size();
        int cc = -1;
        while (p < n) {
            cc = (unsigned char)d[p++];
            if (cc == '>' || cc == '+' || cc == '@') break;
            cc = -1;
            if (d[p - 1] == '\n') continue;
            const size_t e = p - 1;
            void const* q = std::memchr(d + p, '\n', n - p);
            const size_t le = q ? (size_t)((char const*)q - d) : n;
            seq.append(d + e, le - e);
            p = le < n ? le + 1 : n;
        }
        if (cc == '+') return fail();
        if (cc == '>' || cc == '@') last = cc;
        lens.push_back(seq.size() - start);
        if (cc == -1) return true;
    }
}

// One input file inflated and parsed: sequence bytes back to back and one
// length per record.
void read_one(std::string const& path, std::string& seq, std::vector<uint64_t>& lens) {
    std::string raw = slurp(path);
    seq.clear();
    lens.clear();
    seq.reserve(raw.size());
    if (parse_fasta_fast(raw.data(), raw.size(), seq, lens)) return;
    parse_fastx(raw.data(), raw.size(), [&](char const* s, size_t l) {
        seq.append(s, l);
        lens.push_back(l);
    });
}
}  // namespace

void read_files(std::vector<std::string> const& files, size_t first, size_t count,
                uint32_t color_base, uint32_t threads, seq_batch& out) {
    struct per_file {
        std::string seq;
        std::vector<uint64_t> lens;
        uint64_t disk = 0;
    };
    std::vector<per_file> pf(count);
    parallel_for(count, threads, [&](size_t i) {
        std::string const& path = files[first + i];
        std::error_code ec;
        auto sz = std::filesystem::file_size(path, ec);
        pf[i].disk = ec ? 0 : (uint64_t)sz;
        read_one(path, pf[i].seq, pf[i].lens);
    });
    uint64_t total = out.seq.size();
    for (auto const& f : pf) total += f.seq.size();
    out.seq.reserve(total);
    for (size_t i = 0; i < count; ++i) {
        out.seq.insert(out.seq.end(), pf[i].seq.begin(), pf[i].seq.end());
        for (uint64_t l : pf[i].lens) {
            out.off.push_back(out.off.back() + l);
            out.color.push_back(color_base + (uint32_t)i);
        }
        out.input_bytes += pf[i].disk;
    }
}

file_probe probe_file(std::string const& path) {
    std::error_code ec;
    const uint64_t sz = std::filesystem::file_size(path, ec);
    if (ec) throw std::runtime_error("could not open input file: " + path);
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("could not open input file: " + path);
    unsigned char head[2] = {0, 0}, tail[4] = {0, 0, 0, 0};
    file_probe p;
    p.size = sz;
    p.gz = std::fread(head, 1, 2, f) == 2 && head[0] == 0x1f && head[1] == 0x8b;
    p.hint = sz;
    if (p.gz && sz >= 18 && std::fseek(f, -4, SEEK_END) == 0 && std::fread(tail, 1, 4, f) == 4) {
        const uint64_t isize = (uint64_t)tail[0] | ((uint64_t)tail[1] << 8) | ((uint64_t)tail[2] << 16) |
                               ((uint64_t)tail[3] << 24);
        // the size field is mod 2^32: take the largest size congruent to it
        // that deflate's maximum ratio (1032:1) allows
        const uint64_t lim = sz * 1032;
        uint64_t v = isize;
        while (v + (uint64_t(1) << 32) <= lim) v += uint64_t(1) << 32;
        p.hint = v;
    }
    std::fclose(f);
    return p;
}

uint64_t inflated_size_hint(std::string const& path) { return probe_file(path).hint; }

void probe_files(std::vector<std::string> const& files, uint32_t threads, std::vector<file_probe>& out) {
    out.assign(files.size(), file_probe());
    parallel_for(files.size(), threads, [&](size_t i) { out[i] = probe_file(files[i]); });
}

void read_raw_files(std::vector<std::string> const& files, uint32_t threads, char* dst, uint64_t const* off) {
    parallel_for(files.size(), threads, [&](size_t i) {
        const int fd = ::open(files[i].c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("could not open input file: " + files[i]);
        uint64_t a = off[i];
        const uint64_t b = off[i + 1];
        while (a < b) {
            const ssize_t r = ::read(fd, dst + a, (size_t)std::min<uint64_t>(b - a, 1ull << 30));
            if (r <= 0) {
                ::close(fd);
                throw std::runtime_error("short read of input file: " + files[i]);
            }
            a += (uint64_t)r;
        }
        ::close(fd);
    });
}

bool read_files_into(std::vector<std::string> const& files, size_t first, size_t count, uint32_t color_base,
                     uint32_t threads, char* dst, uint64_t cap, seq_batch& out) {
    struct per_file {
        std::string seq;
        std::vector<uint64_t> lens;
        uint64_t disk = 0;
    };
    std::vector<per_file> pf(count);
    parallel_for(count, threads, [&](size_t i) {
        std::string const& path = files[first + i];
        std::error_code ec;
        auto sz = std::filesystem::file_size(path, ec);
        pf[i].disk = ec ? 0 : (uint64_t)sz;
        read_one(path, pf[i].seq, pf[i].lens);
    });
    std::vector<uint64_t> at(count + 1, 0);
    for (size_t i = 0; i < count; ++i) at[i + 1] = at[i] + pf[i].seq.size();
    if (at[count] > cap) return false;
    parallel_for(count, threads, [&](size_t i) {
        if (!pf[i].seq.empty()) std::memcpy(dst + at[i], pf[i].seq.data(), pf[i].seq.size());
    });
    for (size_t i = 0; i < count; ++i) {
        for (uint64_t l : pf[i].lens) {
            out.off.push_back(out.off.back() + l);
            out.color.push_back(color_base + (uint32_t)i);
        }
        out.input_bytes += pf[i].disk;
    }
    return true;
}

range_file::range_file(std::string const& path) : m_path(path) {
    m_fd = ::open(path.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0644);
    if (m_fd < 0) throw std::runtime_error("cannot open output file: " + path + ": " + std::strerror(errno));
    struct statfs fs;
    constexpr long kTmpfsMagic = 0x01021994;
    m_tmpfs = ::fstatfs(m_fd, &fs) == 0 && (long)fs.f_type == kTmpfsMagic;
}

range_file::~range_file() {
    if (m_fd >= 0) ::close(m_fd);
}

void range_file::write(uint8_t const* data, uint64_t off, uint64_t n, uint32_t threads) {
    if (n == 0) return;
    const uint64_t piece = std::max<uint64_t>(32ull << 20, (n + threads - 1) / std::max<uint32_t>(threads, 1));
    const size_t np = (size_t)((n + piece - 1) / piece);
    std::atomic<bool> bad{false};
    void* map = MAP_FAILED;
    const uint64_t pg = (uint64_t)::sysconf(_SC_PAGESIZE);
    const uint64_t a = off & ~(pg - 1);
    if (m_tmpfs && ::fallocate(m_fd, 0, (off_t)off, (off_t)n) == 0)
        map = ::mmap(nullptr, (size_t)(off + n - a), PROT_WRITE, MAP_SHARED, m_fd, (off_t)a);
    if (map != MAP_FAILED) {
        uint8_t* dst = (uint8_t*)map + (off - a);
        parallel_for(np, threads, [&](size_t i) {
            const uint64_t x = i * piece, y = std::min<uint64_t>(n, x + piece);
            std::memcpy(dst + x, data + x, (size_t)(y - x));
        });
        if (::munmap(map, (size_t)(off + n - a)) != 0) bad = true;
    } else {
        parallel_for(np, threads, [&](size_t i) {
            uint64_t x = i * piece;
            const uint64_t y = std::min<uint64_t>(n, x + piece);
            while (x < y) {
                const ssize_t w =
                    ::pwrite(m_fd, data + x, (size_t)std::min<uint64_t>(y - x, 1ull << 30), (off_t)(off + x));
                if (w <= 0) {
                    bad = true;
                    return;
                }
                x += (uint64_t)w;
            }
        });
    }
    if (bad) throw std::runtime_error("short write to " + m_path);
}

void range_file::finish(uint64_t total) {
    const int fd = m_fd;
    m_fd = -1;
    const bool ok = ::ftruncate(fd, (off_t)total) == 0;
    if (::close(fd) != 0 || !ok) throw std::runtime_error("cannot finish output file " + m_path);
}

void write_file_parallel(std::string const& path, uint8_t const* data, uint64_t n, uint32_t threads) {
    range_file f(path);
    f.write(data, 0, n, threads);
    f.finish(n);
}

// ---------------------------------------------------------------- buckets
bucket_file_set::bucket_file_set(std::string dir, uint32_t num_buckets)
    : m_dir(std::move(dir)), m_B(num_buckets), m_files(num_buckets, nullptr), m_unc(num_buckets, 0) {
    std::filesystem::create_directories(m_dir);
    for (uint32_t b = 0; b < m_B; ++b) {
        std::FILE* f = std::fopen(path(b).c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open bucket file: " + path(b) + ": " + std::strerror(errno));
        m_files[b] = f;
    }
}

bucket_file_set::~bucket_file_set() {
    for (void* f : m_files)
        if (f) std::fclose((std::FILE*)f);
}

std::string bucket_file_set::path(uint32_t b) const { return m_dir + "/bucket_" + std::to_string(b) + ".bin"; }

void bucket_file_set::append_frames(uint8_t const* raw, uint64_t const* boff, uint32_t threads) {
    append_frames_range(raw, boff, 0, m_B, threads);
}

void bucket_file_set::append_frames_range(uint8_t const* raw, uint64_t const* boff, uint32_t b_lo, uint32_t b_hi,
                                          uint32_t threads) {
    // One LZ4 frame per bucket slice (records never straddle a frame: the
    // slice is whole records of one device serialization).
    std::vector<uint64_t> comp(b_hi - b_lo, 0);
    parallel_for(b_hi - b_lo, threads, [&](size_t i) {
        const size_t b = b_lo + i;
        const uint64_t a = boff[b], e = boff[b + 1];
        if (a == e) return;
        if (e - a > (uint64_t)LZ4_MAX_INPUT) throw std::runtime_error("bucket slice too large for one LZ4 frame");
        std::FILE* f = (std::FILE*)m_files[b];
        const int src = (int)(e - a);
        std::vector<char>& out = lz4_scratch((size_t)LZ4_compressBound(src));
        int c = LZ4_compress_default((char const*)raw + a, out.data(), src, (int)out.size());
        if (c <= 0) throw std::runtime_error("LZ4_compress_default failed on " + path((uint32_t)b));
        uint32_t u32 = (uint32_t)src, c32 = (uint32_t)c;
        if (std::fwrite(&u32, 4, 1, f) != 1 || std::fwrite(&c32, 4, 1, f) != 1 ||
            std::fwrite(out.data(), 1, (size_t)c, f) != (size_t)c)
            throw std::runtime_error("short write to " + path((uint32_t)b));
        m_unc[b] += (uint64_t)src;
        comp[i] = 8 + (uint64_t)c;
    });
    for (uint64_t c : comp) m_comp += c;
}

void bucket_file_set::close() {
    for (uint32_t b = 0; b < m_B; ++b) {
        std::FILE* f = (std::FILE*)m_files[b];
        if (!f) continue;
        uint32_t eof = 0;
        if (std::fwrite(&eof, 4, 1, f) != 1) throw std::runtime_error("short write to " + path(b));
        std::fclose(f);
        m_files[b] = nullptr;
        m_comp += 4;
    }
}

// ---- stitch round store, round 0
namespace {
constexpr uint64_t ROUND_FRAME = 4ull << 20;  // round_store_file::FRAME_BUDGET (stitch_extmem.hpp:556)

inline uint32_t get_u32(uint8_t const* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
}  // namespace

round0_store::round0_store(std::string dir, uint32_t num_buckets)
    : m_dir(std::move(dir)), m_B(num_buckets), m_files(num_buckets, nullptr), m_pend(num_buckets) {
    std::filesystem::create_directories(m_dir);
    // a round-0 file left from an earlier build would be read as input
    for (uint32_t b = 0; b < m_B; ++b) std::remove(path(b).c_str());
}

round0_store::~round0_store() {
    for (void* f : m_files)
        if (f) std::fclose((std::FILE*)f);
}

std::string round0_store::path(uint32_t b) const {
    return m_dir + "/stitch_r0_b" + std::to_string(b) + ".bin";
}

void round0_store::flush(uint32_t b, uint8_t const* data, uint64_t n, uint64_t& comp) {
    if (n > LZ4_MAX_INPUT) throw std::runtime_error("stitch round frame too large for LZ4");
    std::FILE* f = (std::FILE*)m_files[b];
    if (!f) {
        f = std::fopen(path(b).c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open stitch round file: " + path(b) + ": " + std::strerror(errno));
        m_files[b] = f;
    }
    std::vector<char>& out = lz4_scratch((size_t)LZ4_compressBound((int)n));
    const int c = LZ4_compress_default((char const*)data, out.data(), (int)n, (int)out.size());
    if (c <= 0) throw std::runtime_error("LZ4_compress_default failed on " + path(b));
    const uint32_t u32 = (uint32_t)n, c32 = (uint32_t)c;
    if (std::fwrite(&u32, 4, 1, f) != 1 || std::fwrite(&c32, 4, 1, f) != 1 ||
        std::fwrite(out.data(), 1, (size_t)c, f) != (size_t)c)
        throw std::runtime_error("short write to " + path(b));
    comp += 8 + (uint64_t)c;
}

void round0_store::append(uint8_t const* tigs, uint64_t const* boff, uint32_t threads) {
    append_range(tigs, boff, 0, m_B, threads);
}

void round0_store::append_range(uint8_t const* tigs, uint64_t const* boff, uint32_t b_lo, uint32_t b_hi,
                                uint32_t threads) {
    std::vector<uint64_t> comp(b_hi - b_lo, 0);
    parallel_for(b_hi - b_lo, threads, [&](size_t bi) {
        const uint32_t b = b_lo + (uint32_t)bi;
        const uint64_t a = boff[b], e = boff[b + 1];
        if (a == e) return;
        std::vector<uint8_t>& pend = m_pend[b];
        uint64_t seg = a, pos = a;
        while (pos < e) {
            // ext_tig_serialize layout: 13-byte head, runs, u32 seq_len, 2-bit bases
            if (pos + 13 > e) throw std::runtime_error("truncated tig in round-0 output");
            const uint64_t nruns = get_u32(tigs + pos + 9);
            const uint64_t lp = pos + 13 + 12 * nruns;
            if (lp + 4 > e) throw std::runtime_error("truncated tig in round-0 output");
            pos = lp + 4 + ((uint64_t)get_u32(tigs + lp) + 3) / 4;
            if (pos > e) throw std::runtime_error("truncated tig in round-0 output");
            // emit() appends one tig, then flushes once the batch holds a frame
            if (pend.size() + (pos - seg) >= ROUND_FRAME) {
                if (pend.empty()) {
                    flush(b, tigs + seg, pos - seg, comp[bi]);
                } else {
                    pend.insert(pend.end(), tigs + seg, tigs + pos);
                    flush(b, pend.data(), pend.size(), comp[bi]);
                    pend.clear();
                }
                seg = pos;
            }
        }
        pend.insert(pend.end(), tigs + seg, tigs + e);
    });
    m_raw += boff[b_hi] - boff[b_lo];
    for (uint64_t c : comp) m_comp += c;
}

void round0_store::finish(uint32_t threads) {
    std::vector<uint64_t> comp(m_B, 0);
    parallel_for(m_B, threads, [&](size_t bi) {
        const uint32_t b = (uint32_t)bi;
        std::vector<uint8_t>& pend = m_pend[b];
        if (!pend.empty()) {
            flush(b, pend.data(), pend.size(), comp[b]);
            std::vector<uint8_t>().swap(pend);
        }
        std::FILE* f = (std::FILE*)m_files[b];
        if (!f) return;
        const uint32_t eof = 0;
        if (std::fwrite(&eof, 4, 1, f) != 1) throw std::runtime_error("short write to " + path(b));
        if (std::fclose(f) != 0) throw std::runtime_error("close failed on " + path(b));
        m_files[b] = nullptr;
        comp[b] += 4;
    });
    for (uint64_t c : comp) m_comp += c;
}

namespace {
// The record at p: its end, or 0 when it runs past n.
// [u8 open_flags][u32 nruns][nruns x 12][u32 seq_len][seq]
inline uint64_t frag_record_end(uint8_t const* d, uint64_t n, uint64_t p) {
    if (p + 5 > n) return 0;
    const uint64_t lp = p + 5 + 12ull * get_u32(d + p + 1);
    if (lp + 4 > n) return 0;
    const uint64_t q = lp + 4 + get_u32(d + lp);
    return q > n ? 0 : q;
}

// Could a record start at p?  Flags 0..3, a run count and length that stay in
// the buffer, ACGT bases, and the same for the records after it (4 deep).
bool plausible_start(uint8_t const* d, uint64_t n, uint64_t p) {
    for (int depth = 0; depth < 4 && p < n; ++depth) {
        if (d[p] > 3 || p + 5 > n || get_u32(d + p + 1) > (1u << 20)) return false;
        const uint64_t q = frag_record_end(d, n, p);
        if (!q) return false;
        const uint64_t lp = p + 5 + 12ull * get_u32(d + p + 1);
        const uint64_t s = lp + 4, e = std::min<uint64_t>(q, s + 16);
        for (uint64_t x = s; x < e; ++x)
            if (d[x] != 'A' && d[x] != 'C' && d[x] != 'G' && d[x] != 'T') return false;
        p = q;
    }
    return true;
}
}  // namespace

uint64_t frag_record_offsets(uint8_t const* d, uint64_t n, uint32_t threads,
                             std::function<uint64_t*(uint64_t)> const& alloc,
                             std::vector<std::vector<uint64_t>>* scratch) {
    const uint64_t P = std::max<uint64_t>(1, std::min<uint64_t>(threads, n >> 20));
    // Part t covers [c(t), c(t + 1)).  Part 0 starts at a record; every other
    // part guesses its first record (plausible_start) and follows the chain
    // to the first record at or past its end.  Chains that meet stay together
    // (a record determines the next), so the merge takes a part's chain from
    // where the true chain meets it and walks the true chain itself elsewhere.
    auto c = [&](uint64_t t) { return n * t / P; };
    struct part {
        uint64_t start = 0, end = 0;
        bool found = false, broken = false;
        std::vector<uint64_t> recs;
    };
    std::vector<part> parts(P);
    // the caller's vectors keep their pages from call to call
    if (scratch) {
        scratch->resize(std::max<size_t>(scratch->size(), P));
        for (uint64_t t = 0; t < P; ++t) parts[t].recs.swap((*scratch)[t]);
    }
    struct give_back {
        std::vector<part>& parts;
        std::vector<std::vector<uint64_t>>* scratch;
        ~give_back() {
            if (scratch)
                for (size_t t = 0; t < parts.size(); ++t) parts[t].recs.swap((*scratch)[t]);
        }
    } give_back_{parts, scratch};
    parallel_for(P, (uint32_t)P, [&](size_t t) {
        part& pt = parts[t];
        uint64_t pos = c(t);
        const uint64_t lim = c(t + 1);
        if (t > 0) {
            while (pos < lim && !plausible_start(d, n, pos)) ++pos;
            if (pos >= lim) return;
        }
        pt.found = true;
        pt.start = pos;
        pt.recs.clear();
        pt.recs.reserve((lim - pos) / 64 + 16);
        while (pos < lim) {
            const uint64_t q = frag_record_end(d, n, pos);
            if (!q) {
                pt.broken = true;
                break;
            }
            pt.recs.push_back(pos);
            pos = q;
        }
        pt.end = pos;
    });
    // The merge plan: per part, the records walked here (where the part's own
    // chain was not yet joined) and then the part's chain from the join on.
    struct seg {
        std::vector<uint64_t> const* v;
        size_t a, b;
    };
    std::vector<std::vector<uint64_t>> walked(P);
    std::vector<seg> segs;
    uint64_t e = 0;  // the next true record start
    for (uint64_t t = 0; t < P; ++t) {
        const uint64_t lim = c(t + 1);
        if (e >= lim) continue;  // a record from an earlier part spans this one
        part const& pt = parts[t];
        size_t j = 0;
        if (pt.found) j = std::lower_bound(pt.recs.begin(), pt.recs.end(), e) - pt.recs.begin();
        bool joined = false;
        while (e < lim) {
            while (pt.found && j < pt.recs.size() && pt.recs[j] < e) ++j;
            if (pt.found && j < pt.recs.size() && pt.recs[j] == e) {
                // joined: the rest of this part's chain is true
                if (pt.broken) throw std::runtime_error("truncated fragment record");
                joined = true;
                break;
            }
            const uint64_t q = frag_record_end(d, n, e);
            if (!q) throw std::runtime_error("truncated fragment record");
            walked[t].push_back(e);
            e = q;
        }
        if (!walked[t].empty()) segs.push_back({&walked[t], 0, walked[t].size()});
        if (joined) {
            segs.push_back({&pt.recs, j, pt.recs.size()});
            e = pt.end;
        }
    }
    if (e != n) throw std::runtime_error("truncated fragment record");
    std::vector<uint64_t> at(segs.size() + 1, 0);
    for (size_t i = 0; i < segs.size(); ++i) at[i + 1] = at[i] + (segs[i].b - segs[i].a);
    const uint64_t nrec = at.back();
    uint64_t* out = alloc(nrec + 1);
    parallel_for(segs.size(), threads, [&](size_t i) {
        if (segs[i].b > segs[i].a)
            std::memcpy(out + at[i], segs[i].v->data() + segs[i].a, 8 * (segs[i].b - segs[i].a));
    });
    out[nrec] = n;
    return nrec;
}

void frag_record_offsets(uint8_t const* d, uint64_t n, std::vector<uint64_t>& off, uint32_t threads) {
    frag_record_offsets(d, n, threads, [&](uint64_t m) {
        off.resize(m);
        return off.data();
    });
}

void read_bucket_files(std::string const& dir, uint32_t B, uint32_t threads,
                       std::function<uint8_t*(uint64_t)> const& alloc, bucket_bytes& out,
                       bool delete_after) {
    read_bucket_range(dir, B, 0, B, threads, alloc, out);
    if (delete_after) delete_bucket_files(dir, 0, B);
}

void delete_bucket_files(std::string const& dir, uint32_t b_lo, uint32_t b_hi) {
    for (uint32_t b = b_lo; b < b_hi; ++b) {
        std::error_code ec;
        std::filesystem::remove(dir + "/bucket_" + std::to_string(b) + ".bin", ec);
    }
}

std::vector<uint64_t> bucket_sizes(std::string const& dir, uint32_t B, uint32_t threads) {
    std::vector<uint64_t> unc(B, 0);
    parallel_for(B, threads, [&](size_t b) {
        std::string p = dir + "/bucket_" + std::to_string(b) + ".bin";
        std::FILE* f = std::fopen(p.c_str(), "rb");
        if (!f) return;
        uint32_t hdr[2];
        while (std::fread(hdr, 4, 1, f) == 1 && hdr[0] != 0) {
            if (std::fread(hdr + 1, 4, 1, f) != 1 || std::fseek(f, (long)hdr[1], SEEK_CUR) != 0) {
                std::fclose(f);
                throw std::runtime_error("short read of frame header on " + p);
            }
            unc[b] += hdr[0];
        }
        std::fclose(f);
    });
    return unc;
}

void read_bucket_range(std::string const& dir, uint32_t B, uint32_t b_lo, uint32_t b_hi, uint32_t threads,
                       std::function<uint8_t*(uint64_t)> const& alloc, bucket_bytes& out) {
    struct frame {
        uint32_t u, c;
        long pos;
    };
    std::vector<std::vector<frame>> frames(B);
    std::vector<std::vector<char>> comp(B);
    out.bucket_unc.assign(B, 0);
    // pass 1: read each file of the range whole (compressed), index its frames
    parallel_for(b_hi - b_lo, threads, [&](size_t i) {
        const size_t b = b_lo + i;
        std::string p = dir + "/bucket_" + std::to_string(b) + ".bin";
        std::FILE* f = std::fopen(p.c_str(), "rb");
        if (!f) return;  // a missing bucket file is an empty bucket
        std::fseek(f, 0, SEEK_END);
        long sz = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        comp[b].resize((size_t)sz);
        if (sz > 0 && std::fread(comp[b].data(), 1, (size_t)sz, f) != (size_t)sz) {
            std::fclose(f);
            throw std::runtime_error("short read of " + p);
        }
        std::fclose(f);
        size_t q = 0;
        for (;;) {
            if (q + 4 > comp[b].size()) {
                if (q == comp[b].size()) break;
                throw std::runtime_error("short read of frame header on " + p);
            }
            uint32_t u;
            std::memcpy(&u, comp[b].data() + q, 4);
            q += 4;
            if (u == 0) break;
            if (q + 4 > comp[b].size()) throw std::runtime_error("short read of compressed_size on " + p);
            uint32_t c;
            std::memcpy(&c, comp[b].data() + q, 4);
            q += 4;
            if (q + c > comp[b].size()) throw std::runtime_error("short read of compressed payload on " + p);
            frames[b].push_back({u, c, (long)q});
            q += c;
            out.bucket_unc[b] += u;
        }
    });
    uint64_t total = 0;
    for (uint64_t u : out.bucket_unc) total += u;
    out.nbytes = total;
    out.data = alloc(total + 64);
    std::memset(out.data + total, 0, 64);
    std::vector<uint64_t> bstart(B + 1, 0);
    for (uint32_t b = 0; b < B; ++b) bstart[b + 1] = bstart[b] + out.bucket_unc[b];
    out.chunk_off.clear();
    out.chunk_bucket.clear();
    for (uint32_t b = 0; b < B; ++b) {
        uint64_t o = bstart[b];
        for (auto const& fr : frames[b]) {
            out.chunk_off.push_back(o);
            out.chunk_bucket.push_back(b);
            o += fr.u;
        }
    }
    out.chunk_off.push_back(total);
    // pass 2: decompress in parallel into place
    parallel_for(b_hi - b_lo, threads, [&](size_t i) {
        const size_t b = b_lo + i;
        uint64_t o = bstart[b];
        for (auto const& fr : frames[b]) {
            int d = LZ4_decompress_safe(comp[b].data() + fr.pos, (char*)out.data + o, (int)fr.c, (int)fr.u);
            if (d < 0 || (uint32_t)d != fr.u)
                throw std::runtime_error("LZ4_decompress_safe failed on bucket " + std::to_string(b));
            o += fr.u;
        }
        std::vector<char>().swap(comp[b]);
    });
}

void write_color_sets_ef(std::string const& path, uint32_t C, uint64_t const* words, uint64_t nbits,
                         uint64_t nvalues, uint64_t l, uint64_t const* low, uint64_t const* high,
                         uint64_t high_bits) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open color-set output: " + path);
    const uint32_t st = (uint32_t)(0.25 * C), dt = (uint32_t)(0.75 * C);
    const uint64_t nwords = (nbits + 63) / 64;
    bool ok = std::fwrite(&C, 4, 1, f) == 1 && std::fwrite(&st, 4, 1, f) == 1 &&
              std::fwrite(&dt, 4, 1, f) == 1 && std::fwrite(&nbits, 8, 1, f) == 1 &&
              std::fwrite(&nwords, 8, 1, f) == 1;
    if (ok && nwords) ok = std::fwrite(words, 8, nwords, f) == nwords;
    const uint64_t U = nbits, lbits = nvalues * l, lw = (lbits + 63) / 64, hw = (high_bits + 63) / 64;
    ok = ok && std::fwrite(&U, 8, 1, f) == 1 && std::fwrite(&nvalues, 8, 1, f) == 1 && std::fwrite(&l, 8, 1, f) == 1;
    ok = ok && std::fwrite(&lbits, 8, 1, f) == 1 && std::fwrite(&lw, 8, 1, f) == 1;
    if (ok && lw) ok = std::fwrite(low, 8, lw, f) == lw;
    ok = ok && std::fwrite(&high_bits, 8, 1, f) == 1 && std::fwrite(&hw, 8, 1, f) == 1;
    if (ok && hw) ok = std::fwrite(high, 8, hw, f) == hw;
    std::fclose(f);
    if (!ok) throw std::runtime_error("short write to " + path);
}

}  // namespace io
}  // namespace cdbg
