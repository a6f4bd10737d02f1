#pragma once
// Recording stand-in for the reference's phase1_bucket_write/bucket_io.hpp,
// used only by oracle/ref_harness/ref_phase1.cpp.  It sits earlier on the
// include path than the reference's include/ directory, so the reference's
// bucket_ingester.hpp (emit_super_kmers, ingest_file_bucketed) compiles
// unmodified against it and every super-k-mer it emits through
// per_thread_bucket_buffers::append (bucket_io.hpp:617) is recorded instead of
// compacted.  bucket_prof()/bucket_write_prof come from the reference's real
// util.hpp.

#include <cstdint>
#include <cstdio>
#include <unordered_map>  // util.hpp uses it without including it
#include <vector>

#include "phase1_bucket_write/super_kmer.hpp"
#include "util.hpp"

namespace cdbg {

struct bucket_writer {};

// One emitted super-k-mer occurrence.
struct recorded_super {
    uint32_t bucket;
    uint8_t flags;
    uint32_t color;
    std::vector<uint8_t> bases;  // 0..3 per base
};

inline std::vector<recorded_super>& recorded_supers() {
    static std::vector<recorded_super> v;
    return v;
}

struct per_thread_bucket_buffers {
    explicit per_thread_bucket_buffers(bucket_writer&) {}
    void append(uint32_t b, uint8_t flags, uint32_t color, uint8_t const* sk_bases, uint32_t len) {
        recorded_supers().push_back(
            {b, (uint8_t)(flags & 0xfu), color, std::vector<uint8_t>(sk_bases, sk_bases + len)});
    }
    void flush_all() {}
};

}  // namespace cdbg
