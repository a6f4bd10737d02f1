// Phase 1 (bucket-write) on the device: data structures and entry points.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.cuh"

namespace cdbg {

// Input sequences (device pointers): ASCII bytes of all sequences back to
// back, seq_off[num_seqs + 1] byte offsets, one color per sequence.
struct seq_input {
    uint8_t const* ascii;
    uint64_t nbytes;
    uint64_t const* seq_off;
    uint32_t const* seq_color;
    uint32_t num_seqs;
};

// ACGT runs of length >= k packed into one 2-bit stream (device).
struct run_table {
    uint32_t n = 0;
    uint64_t* src = nullptr;   // byte offset of the run in the ASCII input
    uint32_t* len = nullptr;   // bases
    uint32_t* color = nullptr;
    uint64_t* soff = nullptr;  // stream base offset (multiple of 32)
    uint64_t* words = nullptr; // 2-bit stream, base i at bits 2*(i%32) of word i/32
    uint64_t nwords = 0;
    uint64_t n_kmers = 0;      // sum over runs of (len - k + 1)
    uint64_t n_bases = 0;      // sum over runs of len
};

// Super-k-mer records grouped by bucket (device).  Record bases live in a
// 2-bit stream `words` at base position start[r].
struct record_set {
    uint32_t B = 0;
    uint64_t n = 0;
    uint64_t* start = nullptr;
    uint32_t* len = nullptr;
    uint32_t* flags = nullptr;     // SK flag bits 0..3
    uint64_t* col_off = nullptr;   // n + 1 entries
    uint32_t* colors = nullptr;    // ascending per record
    uint64_t ncolors = 0;
    uint64_t* bucket_start = nullptr;  // B + 1 record offsets
    uint64_t const* words = nullptr;
    uint64_t nwords = 0;
    uint64_t n_occ_supers = 0;     // super-k-mer occurrences before dedup
};

struct phase1_stats {
    uint64_t n_runs, n_bases, n_kmers, n_supers, n_records, n_colors;
};

// Runs + packing: ASCII -> 2-bit stream of ACGT runs >= k.
// The 2-bit stream (rt.words) comes from `out`, everything else from A.  With
// `words_out`, the runs are packed at word `word_base` of that stream instead
// (capacity `words_cap` words) and rt.soff / rt.words / rt.nwords refer to it.
void build_runs(seq_input const& in, uint32_t k, dev_arena& A, cudaStream_t st, run_table& rt, dev_arena& out,
                uint64_t* words_out = nullptr, uint64_t word_base = 0, uint64_t words_cap = 0);

// Super-k-mer occurrences of every run (for parity tests): arrays in input
// order, allocated from the arena.  Returns the count.
struct super_list {
    uint64_t n = 0;
    uint64_t* start = nullptr;
    uint32_t* len = nullptr;
    uint32_t* color = nullptr;
    uint32_t* flags = nullptr;
    uint32_t* bucket = nullptr;
    uint64_t* key = nullptr;
    // packed form (start, len, color << 4 | flags) instead of the arrays above
    uint4* packed = nullptr;
};
// `tile` = (k-1)-mers per minimizer tile: 1024 or 2048 (0 = 2048).  With
// `packed` (for build_records; colors must be < 2^28) only `key` and
// `packed` are filled.
void find_supers(run_table const& rt, uint32_t k, uint32_t m, uint32_t B, dev_arena& A,
                 cudaStream_t st, super_list& out, uint32_t* d_err, uint32_t tile = 0, bool packed = false);

// Keep only the super-k-mers of buckets [lo, hi) (input order kept), in new
// arrays from A: one rank's share of a build split by bucket range.
void keep_bucket_range(super_list& sl, uint32_t B, uint32_t lo, uint32_t hi, dev_arena& A, cudaStream_t st);

// Dedup super-k-mers into canonical bucket records.
// Record arrays come from `out`, temporaries from A.
void build_records(run_table const& rt, super_list& sl, uint32_t k, uint32_t B, dev_arena& A,
                   cudaStream_t st, record_set& rs, uint32_t* d_err, dev_arena& out);

// Serialized record bytes (reference record layout, super_kmer.hpp:105-117):
// out bytes for all buckets back to back, bucket_bytes[B + 1] offsets (device).
struct serialized_buckets {
    uint8_t* bytes = nullptr;
    uint64_t nbytes = 0;
    uint64_t* bucket_off = nullptr;  // B + 1, device
    uint64_t* rec_off = nullptr;     // n + 1, device
};
void serialize_records(record_set const& rs, dev_arena& A, cudaStream_t st, serialized_buckets& out);

// Sum of the serialized sizes of all records (reference record layout) into
// the device word *d_sum, without synchronizing.
void record_bytes_async(record_set const& rs, unsigned long long* d_sum, cudaStream_t st);

// Parse serialized bucket bytes (device, 8-byte aligned, padded) into a
// record_set.  chunk_off[nchunks + 1] are byte offsets where a record starts
// (bucket and LZ4-frame starts); chunk_bucket[nchunks] the bucket of each.
void parse_records(uint8_t const* bytes, uint64_t nbytes, uint64_t const* chunk_off,
                   uint32_t const* chunk_bucket, uint32_t nchunks, uint32_t B, dev_arena& A,
                   cudaStream_t st, record_set& rs, uint32_t* d_err);

}  // namespace cdbg
