// gzip inflate and FASTA record compaction on the device: the input side of
// phase 1 for collections of many compressed genomes (one file per color).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "arena.cuh"
#include "common.cuh"

namespace cdbg {

// Per-stream outcome.  Anything but STREAM_OK sends the whole call back to the
// host reader, which then decides with zlib and the kseq rules.
enum stream_status : uint32_t {
    STREAM_OK = 0,
    STREAM_OVERFLOW = 1,  // inflated past its region (e.g. a multi-member file)
    STREAM_BAD = 2,       // not a gzip stream this inflater accepts
    STREAM_FASTQ = 3,     // a FASTQ record ('@' header or '+' line)
};

// One stream per input file, all arrays on the device.  Stream f reads
// in[in_off[f], in_off[f] + in_len[f]) -- gzip members back to back when
// gz[f], else plain bytes -- and writes region out[out_off[f], out_off[f] +
// out_cap[f]) (out_off 16-byte aligned).  `in` must stay readable for 64
// bytes past the last stream.
struct stream_set {
    uint8_t const* in;
    uint64_t const* in_off;
    uint64_t const* in_len;
    uint8_t const* gz;
    uint8_t* out;
    uint64_t const* out_off;
    uint64_t const* out_cap;
    uint64_t* out_len;   // bytes produced
    uint32_t* status;    // stream_status
    uint32_t n;
};

// Inflates (or copies) every stream into its region.
void inflate_streams(stream_set const& s, cudaStream_t st);

// Rewrites each STREAM_OK region in place as its FASTA records' sequence
// bytes, each header line replaced by its '>' (not a base, so runs of bases
// end at record boundaries), and fills the rest of the region (up to
// out_cap rounded up to 16 bytes) with '\n'.  seq_bytes[f] = sequence bytes
// kept (without the '>' separators).  Sets STREAM_FASTQ for FASTQ input.
void fasta_compact(stream_set const& s, uint64_t* seq_bytes, cudaStream_t st);

}  // namespace cdbg
