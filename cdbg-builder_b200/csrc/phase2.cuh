// Phase 2 (bucket-process) on the device: entry point and outputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "arena.cuh"
#include "phase1.cuh"

namespace cdbg {

// Device storage that outlives one build (kept by the engine so repeated
// builds reuse it): the color-class dictionary and the device-resident frag
// bytes.  After a build with outputs left on the device, words/bit_off/frag
// hold that build's .color_sets words, class offsets and frag spill.
struct phase2_state {
    dvec<uint64_t> cls_hash;   // per class: 64-bit set hash
    dvec<uint64_t> bit_off;    // per class: bit offset (n + 1 entries)
    dvec<uint64_t> words;      // encoded classes
    dvec<uint64_t> slot_hash;  // open-addressing table hash -> class
    dvec<uint32_t> slot_cid;
    dvec<uint8_t> frag;        // frag spill bytes (device-resident builds)
    dvec<uint64_t> frag_off;   // their record offsets (phase2_params::keep_frag_offsets)
    // dictionary size, kept so that a later call can continue it
    uint64_t n = 0, nbits = 0, total_integers = 0, mask = 0;
    // Order later frees on `st` (after a stream switch).
    void set_stream(cudaStream_t st) {
        cls_hash.st_last = bit_off.st_last = words.st_last = slot_hash.st_last = st;
        slot_cid.st_last = st;
        frag.st_last = frag_off.st_last = st;
    }
    void release() {
        cls_hash.release();
        bit_off.release();
        words.release();
        slot_hash.release();
        slot_cid.release();
        frag.release();
        frag_off.release();
    }
    size_t bytes() const {
        return cls_hash.bytes() + bit_off.bytes() + words.bytes() + slot_hash.bytes() + slot_cid.bytes() +
               frag.bytes() + frag_off.bytes();
    }
};

// Outputs of phase 2, accumulated over bucket batches.
struct phase2_result {
    uint64_t frag_host_copied = 0;  // leading frag bytes queued to params.frag_host
    uint64_t words_host_copied = 0; // leading class words queued to params.words_host
    uint64_t offs_host_copied = 0;  // leading class offsets queued to params.offs_host
    // frag_unitigs.bin bytes (unitig_spill.hpp:642-665 record layout), in
    // bucket order and, per bucket, in seed order.
    std::vector<uint8_t> frag;          // host copy (when to_host)
    uint8_t* d_frag = nullptr;          // device copy (when !to_host), arena memory
    uint64_t frag_nbytes = 0;
    // color classes in global cid order
    std::vector<uint64_t> words;        // encoded .color_sets bit vector
    std::vector<uint64_t> offsets;      // bit offset of each class
    uint64_t* d_words = nullptr;        // device copies (when !to_host)
    uint64_t* d_offsets = nullptr;
    uint64_t nbits = 0;
    uint64_t n_classes = 0;
    uint64_t total_integers = 0;
    // persistent storage to use (required when !to_host: the device
    // outputs live in it); null = temporary storage for this call
    phase2_state* state = nullptr;
    // counters
    uint64_t n_occ = 0, n_distinct = 0, n_fragments = 0, total_seq_bytes = 0;
    uint64_t n_multi = 0;
    double ms_device = 0;
};

struct phase2_params {
    uint32_t k = 31;
    uint32_t num_colors = 0;
    uint64_t batch_occ = 0;   // k-mer occurrences per batch (0 = auto)
    bool to_host = true;      // copy outputs to host vectors
    // multi-record color unions as C-bit bitmaps (else as lists; bitmaps cost
    // C/8 bytes per such k-mer, so very large color counts use lists)
    bool union_bitmaps = true;
    // records with at least this many colors get a precomputed bitmap in
    // multi-record unions (performance only)
    uint32_t heavy_colors = 64;
    // k-mer table slots per 4 occurrences of a bucket, 5..16 (performance only)
    uint32_t table_slots_q = 8;
    // continue the class dictionary of the previous call on the same state
    // (bucket ranges of one build processed call by call) instead of
    // starting it empty
    bool keep_dict = false;
    // with to_host: copy the dictionary's words and offsets to the host
    // (the last call of a range-by-range build only)
    bool copy_dict = true;
    // table bytes of one bucket group: the buckets of a batch are processed in
    // groups whose tables fit in this size (performance only; a bucket whose
    // table alone is larger forms a group of its own; the default is one group
    // per batch)
    uint64_t group_bytes = ~0ull;
    // Device-resident mode: fragment bytes of each batch are also copied to
    // this pinned host buffer on `copy_st` while later batches run, as long
    // as they fit in `frag_host_cap` (nothing is streamed when null).
    uint8_t* frag_host = nullptr;
    uint64_t frag_host_cap = 0;
    // called on the host right after a batch's fragment bytes [off, off + n)
    // are queued to frag_host on copy_st (a consumer may write them out while
    // later batches run)
    void (*on_frag)(void* ctx, uint64_t off, uint64_t n) = nullptr;
    void* on_frag_ctx = nullptr;
    // Device-resident mode: also keep the byte offset of every fragment
    // record in phase2_state::frag_off (for a device pass over the records,
    // such as the stitch's round-0 seed).
    bool keep_frag_offsets = false;
    // likewise the class dictionary's completed bit-vector words and class
    // offsets (capacities in entries)
    uint64_t* words_host = nullptr;
    uint64_t words_host_cap = 0;
    uint64_t* offs_host = nullptr;
    uint64_t offs_host_cap = 0;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t copy_ev = nullptr;
};

// Elias-Fano encoding of the class bit offsets plus the total bit count, the
// finalize step of the .color_sets file (streaming_color_set_dict.hpp:221-294):
// n = nclasses + 1 values, l low bits each (l = floor(log2(U / n)) when
// U > n, else 0), value i sets bit (v >> l) + i of the high vector.  Device
// arrays from the arena.
struct ef_encoded {
    uint64_t n = 0, l = 0, high_bits = 0, low_words = 0, high_words = 0;
    uint64_t* low = nullptr;
    uint64_t* high = nullptr;
};
void ef_encode(uint64_t const* d_offsets, uint64_t nclasses, uint64_t total_bits, dev_arena& A, cudaStream_t st,
               ef_encoded& out);

// Run phase 2 over all buckets of `rs` (records grouped by bucket).
void run_phase2(record_set const& rs, phase2_params const& p, dev_arena& A, cudaStream_t st,
                uint32_t* d_err, phase2_result& out);

}  // namespace cdbg
