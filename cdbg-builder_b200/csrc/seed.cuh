// Round 0 of the phase-3 stitch on the device: fragments (frag_unitigs.bin
// records) in, round-store tigs grouped by bucket and the closed fragments'
// monochromatic unitigs out.  The reference seeds round 0 one fragment at a
// time on host threads (phase3_stitch/stitch_extmem.hpp:930-944 ext_seed_one,
// :1013-1099 ext_seed_round0_raw_par).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.cuh"

namespace cdbg {

struct seed_config {
    uint32_t k = 31;
    uint32_t num_buckets = 1024;  // round-store buckets
    bool wide = false;            // 128-bit k-mer words (the reference's CDBG_LARGE_K build)
};

// Device outputs of one seeded range of fragments (memory from the arena).
struct seed_device_out {
    uint8_t* tigs = nullptr;         // serialized tigs, bucket by bucket, fragment order within a bucket
    uint64_t tig_bytes = 0;
    uint64_t* bucket_off = nullptr;  // num_buckets + 1 byte offsets into tigs
    uint8_t* closed = nullptr;       // frag records of the closed unitigs, fragment order
    uint64_t closed_bytes = 0;
    uint64_t n_routed = 0;           // open fragments (tigs)
    uint64_t n_closed = 0;           // closed fragments
    uint64_t n_pieces = 0;           // unitigs in `closed`
    uint64_t routed_record_bytes = 0;  // frag record bytes of the open fragments
};

// frags: device bytes of n records back to back with 8 readable bytes past
// the last; rec_off: n + 1 device byte offsets (rec_off[n] = end).  Malformed
// records (a length that disagrees with rec_off, an open fragment shorter
// than k, a base outside ACGT at a boundary k-mer) set ERR_BAD_RECORD in
// d_err and the call throws.
void seed_fragments(uint8_t const* frags, uint64_t const* rec_off, uint64_t n, seed_config const& c, dev_arena& A,
                    cudaStream_t st, uint32_t* d_err, seed_device_out& out);

}  // namespace cdbg
