// Host-side I/O for the GPU phases: FASTA/FASTQ(.gz) reading, LZ4-framed
// bucket files, the frag spill and the .color_sets file.  Plain C++17 over
// zlib and the system LZ4 block library.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace cdbg {
namespace io {

// Sequences of many files back to back: seq bytes, per-sequence offsets
// (num_seqs + 1) and colors.
struct seq_batch {
    std::vector<char> seq;
    std::vector<uint64_t> off{0};
    std::vector<uint32_t> color;
    uint64_t input_bytes = 0;  // on-disk bytes of the files read
};

// Parse one FASTA/FASTQ buffer with the record rules of kseq_read
// (external/kseq.h, __KSEQ_READ), calling emit(seq_ptr, len) per record.
// Returns false when a FASTQ quality string is truncated (kseq returns -2 and
// the reference's seq_reader::next stops reading the file there).
bool parse_fastx(char const* d, size_t n, std::function<void(char const*, size_t)> const& emit);

// Inflate a file (gzip or plain; gzread passes plain files through).
std::string slurp(std::string const& path);

// Read files [first, first + count) with `threads` threads; file i gets color
// color_base + (i - first).  Throws on an unreadable file.
void read_files(std::vector<std::string> const& files, size_t first, size_t count,
                uint32_t color_base, uint32_t threads, seq_batch& out);

// Upper bound of the bytes inflating `path` yields: the gzip trailer's size
// field for a gzip file (exact for a single-member file under 4 GiB), the
// file size for a plain one.  A multi-member gzip file can exceed it; callers
// that size buffers from it check what they read.
uint64_t inflated_size_hint(std::string const& path);

// What the device reader needs to know about an input file before reading it:
// its size on disk, whether it is gzip, and its inflated size hint.
struct file_probe {
    uint64_t size = 0;
    bool gz = false;
    uint64_t hint = 0;
};
file_probe probe_file(std::string const& path);
void probe_files(std::vector<std::string> const& files, uint32_t threads, std::vector<file_probe>& out);

// Reads files[i] whole (as stored on disk) into dst + off[i], in parallel;
// off has files.size() + 1 entries, off[i + 1] - off[i] the file's size.
void read_raw_files(std::vector<std::string> const& files, uint32_t threads, char* dst, uint64_t const* off);

// read_files with the sequence bytes written to dst[0 .. cap) (out.seq stays
// empty; out.off / out.color / out.input_bytes as read_files).  Returns false,
// with nothing written past cap, when the sequences need more than cap bytes.
bool read_files_into(std::vector<std::string> const& files, size_t first, size_t count, uint32_t color_base,
                     uint32_t threads, char* dst, uint64_t cap, seq_batch& out);

// Write n bytes to `path` with `threads` threads (range_file).
void write_file_parallel(std::string const& path, uint8_t const* data, uint64_t n, uint32_t threads);

// An output file written range by range, in any order, each range by several
// threads: on a RAM-backed file system (tmpfs), where writes to one file take
// its lock one call at a time, through shared mappings of the range filled in
// parallel (the space reserved first, so a full file system is an error, not
// a fault); elsewhere by positional writes of disjoint pieces.
class range_file {
public:
    explicit range_file(std::string const& path);
    ~range_file();
    range_file(range_file const&) = delete;
    range_file& operator=(range_file const&) = delete;
    void write(uint8_t const* data, uint64_t off, uint64_t n, uint32_t threads);
    // sets the file's size and closes it
    void finish(uint64_t total);

private:
    std::string m_path;
    int m_fd = -1;
    bool m_tmpfs = false;
};

// ---- bucket files (bucket_io.hpp:19-40) ------------------------------------
// Append one LZ4 frame per non-empty bucket slice to open bucket files.
class bucket_file_set {
public:
    bucket_file_set(std::string dir, uint32_t num_buckets);
    ~bucket_file_set();
    std::string path(uint32_t b) const;
    // raw: serialized records of all buckets; boff: B + 1 byte offsets.
    void append_frames(uint8_t const* raw, uint64_t const* boff, uint32_t threads);
    // The same for buckets [b_lo, b_hi) only (raw + boff[b] is bucket b's slice).
    void append_frames_range(uint8_t const* raw, uint64_t const* boff, uint32_t b_lo, uint32_t b_hi,
                             uint32_t threads);
    // EOF markers, close; returns per-bucket uncompressed bytes.
    void close();
    std::vector<uint64_t> const& unc_bytes() const { return m_unc; }
    uint64_t comp_bytes() const { return m_comp; }

private:
    std::string m_dir;
    uint32_t m_B;
    std::vector<void*> m_files;
    std::vector<uint64_t> m_unc;
    uint64_t m_comp = 0;
};

// ---- stitch round store, round 0 (stitch_extmem.hpp:471-600) --------------
// <dir>/stitch_r0_b<b>.bin written as the reference's round_store_file writes
// round 0: serialized tigs go to a per-bucket batch that is flushed as one
// LZ4 frame [u32 raw][u32 compressed][bytes] as soon as it holds 4 MiB or
// more, and at finish the rest is flushed and a [u32 0] end mark written.  A
// bucket that received no tig has no file.
class round0_store {
public:
    round0_store(std::string dir, uint32_t num_buckets);
    ~round0_store();
    round0_store(round0_store const&) = delete;
    round0_store& operator=(round0_store const&) = delete;
    std::string path(uint32_t b) const;
    // tigs: serialized tigs, bucket by bucket; boff: num_buckets + 1 offsets.
    // Successive calls append in order (the tigs of one call follow those of
    // the calls before in every bucket).
    void append(uint8_t const* tigs, uint64_t const* boff, uint32_t threads);
    // The same for buckets [b_lo, b_hi) only (tigs + boff[b] is bucket b's).
    void append_range(uint8_t const* tigs, uint64_t const* boff, uint32_t b_lo, uint32_t b_hi, uint32_t threads);
    void finish(uint32_t threads);
    uint64_t raw_bytes() const { return m_raw; }
    uint64_t comp_bytes() const { return m_comp; }

private:
    void flush(uint32_t b, uint8_t const* data, uint64_t n, uint64_t& comp);
    std::string m_dir;
    uint32_t m_B;
    std::vector<void*> m_files;
    std::vector<std::vector<uint8_t>> m_pend;
    uint64_t m_raw = 0, m_comp = 0;
};

// Byte offsets of the records of a frag_unitigs.bin buffer, found by
// `threads` threads: written to alloc(records + 1) (the last = n_bytes); the
// number of records is returned.  Throws at a record that runs past the end.
// `scratch` (optional) holds the threads' lists between calls, so their
// memory is reused.
uint64_t frag_record_offsets(uint8_t const* data, uint64_t n_bytes, uint32_t threads,
                             std::function<uint64_t*(uint64_t)> const& alloc,
                             std::vector<std::vector<uint64_t>>* scratch = nullptr);
// The same into a vector.
void frag_record_offsets(uint8_t const* data, uint64_t n_bytes, std::vector<uint64_t>& off, uint32_t threads);

// Decompressed contents of bucket files 0..B-1 back to back (buffer from
// `alloc`), with `chunk_off` = byte offsets of frame starts (records never
// straddle a frame) and `chunk_bucket` = the bucket of each chunk.
struct bucket_bytes {
    uint8_t* data = nullptr;
    uint64_t nbytes = 0;
    std::vector<uint64_t> chunk_off;   // nchunks + 1
    std::vector<uint32_t> chunk_bucket;
    std::vector<uint64_t> bucket_unc;  // B
};
void read_bucket_files(std::string const& dir, uint32_t B, uint32_t threads,
                       std::function<uint8_t*(uint64_t)> const& alloc, bucket_bytes& out,
                       bool delete_after);
// The same for buckets [b_lo, b_hi) only (bucket_unc still has B entries,
// zero outside the range; chunk_bucket holds absolute bucket numbers).
void read_bucket_range(std::string const& dir, uint32_t B, uint32_t b_lo, uint32_t b_hi, uint32_t threads,
                       std::function<uint8_t*(uint64_t)> const& alloc, bucket_bytes& out);
// Uncompressed bytes of every bucket file, from its frame headers only.
std::vector<uint64_t> bucket_sizes(std::string const& dir, uint32_t B, uint32_t threads);
// Remove bucket files [b_lo, b_hi).
void delete_bucket_files(std::string const& dir, uint32_t b_lo, uint32_t b_hi);

// ---- .color_sets finalize layout (streaming_color_set_dict.hpp:221-294) ----
// header [u32 C][u32 floor(.25C)][u32 floor(.75C)][u64 bits][u64 words],
// the words, then Elias-Fano of the class bit offsets plus the total, in the
// layout of this project's `bits` stand-in (u64 universe, u64 n, u64 l, then
// the low and high bit vectors each as [u64 num_bits][u64 num_words][words]),
// the encoding made on the device (ef_encode): l low bits per value, the low
// and high bit vectors as words.
void write_color_sets_ef(std::string const& path, uint32_t C, uint64_t const* words, uint64_t nbits,
                         uint64_t nvalues, uint64_t l, uint64_t const* low, uint64_t const* high,
                         uint64_t high_bits);

}  // namespace io
}  // namespace cdbg
