/* C-ABI of the B200 (sm_100a) implementation of cdbg-builder's phase 1
 * (bucket-write) and phase 2 (bucket-process).
 *
 * Plain pointers and sizes only.  Every function returns 0 on success and a
 * negative code on failure; cdbg_last_error() then describes the failure
 * (thread-local).  The reference throws std::runtime_error in the same
 * situations (bucket_io.hpp:255-272, 681-699; seq_reader.hpp:48); a C++
 * adapter on the caller's side turns a non-zero return back into that
 * exception.
 *
 * Reference interfaces replaced (paths relative to the reference repository):
 *   cdbg_gpu_phase1  <- ingest_bucketed(files, k, m, B, bucket_writer&, T, ...)
 *                       include/phase1_bucket_write/bucket_ingester.hpp:183-215,
 *                       plus bucket_writer::close() (bucket_io.hpp:389-415) that
 *                       builder.hpp:195 calls right after it.
 *   cdbg_gpu_phase2  <- process_buckets(writer, k, num_colors, T, sink,
 *                       global_dict, mu, done, mem_budget, delete_consumed)
 *                       include/phase2_bucket_process/bucket_walker.hpp:607-779
 *                       with frag_unitig_writer::write_batch as the sink
 *                       (unitig_spill.hpp:491-522) and
 *                       streaming_color_set_dict::intern_with_hashes as the
 *                       color-set merge (streaming_color_set_dict.hpp:148-182).
 *   cdbg_gpu_build   <- the two calls above back to back, in memory (no bucket
 *                       files): builder.hpp:180 + :269.
 *   cdbg_gpu_stitch_seed <- detail::ext_seed_round0_raw_par(for_each_raw,
 *                       frag_record_parse, k, store, sink, done, T), the
 *                       round-0 half of stitch_unitigs_extmem_file_streaming
 *                       (include/phase3_stitch/stitch_extmem.hpp:1013-1099,
 *                       :1120-1129) with a round_store_file as the store.
 */
#ifndef CDBG_GPU_H
#define CDBG_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CDBG_GPU_VERSION 1

typedef struct cdbg_engine cdbg_engine;

/* Engine: one CUDA device, one stream, a cached device arena.  Not
 * thread-safe: one host thread drives one engine. */
int cdbg_engine_create(int device, cdbg_engine** out);
void cdbg_engine_destroy(cdbg_engine* e);
const char* cdbg_last_error(void);
int cdbg_gpu_version(void);

/* Run all work of the engine on a caller-owned CUDA stream (a cudaStream_t
 * passed as void*; NULL restores the engine's own stream), so the caller can
 * bracket calls with its own CUDA events.  No counterpart in the reference
 * (CPU only); measurement plumbing. */
int cdbg_engine_set_stream(cdbg_engine* e, void* stream);

/* Performance knobs of an engine; none changes any output.  Zero fields
 * take the defaults. */
typedef struct cdbg_tuning {
    uint64_t batch_occ;        /* phase-2 k-mer occurrences per bucket batch: the
                                  threshold at which consecutive buckets split
                                  into another batch (0 = from free HBM) */
    uint32_t minimizer_tile;   /* (k-1)-mers per minimizer tile: 1024, 2048 or
                                  4096 (default 4096) */
    uint32_t heavy_colors;     /* records with >= this many colors get a bitmap
                                  in multi-record unions (default 64) */
    uint32_t table_slots_q;    /* k-mer table slots per 4 occurrences of a
                                  bucket, 5..16 (default 8: a load factor of at
                                  most 1/2 over occurrences; fewer slots move
                                  fewer table bytes, longer probes) */
    uint32_t union_lists;      /* 1: multi-record color unions as sorted color
                                  lists, the path taken above 8192 colors
                                  (0 = C-bit bitmaps while C <= 8192) */
    uint32_t table_group_mb;   /* k-mer table MiB per bucket group: a batch's
                                  buckets are processed in groups of at most
                                  this many table bytes, each built, numbered
                                  and probed while cache-resident (0, the
                                  default: one group per batch) */
    uint32_t radix_bits;       /* radix sort digit width: 8 or 11 (default 8) */
    uint32_t gpu_inflate;      /* input files of cdbg_gpu_build_files and
                                  cdbg_gpu_phase1 read by the device (one warp
                                  inflates each gzip file, FASTA records are
                                  cut on the device): 0 (default) when the
                                  work spreads over many files, 1 whenever
                                  the files are gzip, 2 never.  Streams the
                                  device reader does not take (FASTQ, a
                                  multi-member file over its size hint, data
                                  it refuses) send the call to the host
                                  reader; outputs are the same either way. */
} cdbg_tuning;

int cdbg_engine_set_tuning(cdbg_engine* e, const cdbg_tuning* t);
int cdbg_engine_get_tuning(cdbg_engine* e, cdbg_tuning* t);

/* Kernel launches issued by this library in this process so far. */
uint64_t cdbg_launch_count(void);

/* Cap the device memory the engine holds during its calls (arenas + class
 * dictionary; 0 = no cap).  Phase 2 sizes its bucket batches to fit; work
 * that cannot fit fails with an error instead of exceeding the cap.  The
 * engine's share of the reference's -g budget (builder.hpp:258-267). */
int cdbg_engine_set_memory_limit(cdbg_engine* e, uint64_t bytes);

/* Device bytes the engine holds now and at peak since the previous call of
 * this function (which restarts the peak). */
int cdbg_engine_memory(cdbg_engine* e, uint64_t* reserved, uint64_t* peak);

/* Give the engine's cached device memory back to the device's memory pool
 * (stream-ordered, no device-wide synchronization), where other engines can
 * take it.  Invalidates device pointers from its previous builds. */
int cdbg_engine_trim(cdbg_engine* e);

/* Per-kernel device time (CUDA events around each launch on the launching
 * stream): enable = 1 starts collecting (and clears), 0 stops.  Stats copy
 * up to `cap` kernels: NUL-separated names into `names`, total ms and
 * launches; the return value is the number of kernels (or < 0). */
int cdbg_engine_profile(cdbg_engine* e, int32_t enable);
int cdbg_engine_kernel_stats(cdbg_engine* e, char* names, uint64_t names_cap, double* ms,
                             uint64_t* launches, uint32_t cap);
/* Algorithmic bytes (data a launch must read and write, without probes,
 * re-reads or extra passes) summed per kernel over the profiled launches,
 * for the kernels whose launch sites declare them; same name layout. */
int cdbg_engine_kernel_bytes(cdbg_engine* e, char* names, uint64_t names_cap, double* bytes, uint32_t cap);

/* Sequences of many inputs back to back: seq[seq_off[i] .. seq_off[i+1]) is
 * sequence i (ASCII; A/C/G/T in either case are bases, anything else splits
 * runs), of color seq_color[i].  With on_device = 1 all three pointers are
 * device pointers (inputs already resident in HBM). */
typedef struct cdbg_seq_batch {
    const char* seq;
    uint64_t seq_bytes;
    const uint64_t* seq_off; /* num_seqs + 1 */
    const uint32_t* seq_color;
    uint32_t num_seqs;
    int32_t on_device;
} cdbg_seq_batch;

/* Host reader: FASTA/FASTQ (optionally gzip) files -> one sequence batch,
 * file i = color first_color + i, with the record rules of kseq_read
 * (external/kseq.h) that the reference's seq_reader::next uses
 * (phase1_bucket_write/seq_reader.hpp:66).  The buffers belong to the
 * library until cdbg_free_sequences. */
int cdbg_read_sequences(const char* const* files, uint32_t num_files, uint32_t first_color,
                        uint32_t host_threads, cdbg_seq_batch* out);
void cdbg_free_sequences(cdbg_seq_batch* b);

/* ---- phase 1 ------------------------------------------------------------ */

typedef struct cdbg_phase1_args {
    const char* const* files; /* file i = color first_color + i (FASTA/FASTQ, optionally gzip) */
    uint32_t num_files;
    uint32_t k;               /* <= 63 */
    uint32_t m;               /* 0 = compute_best_m(k) (minimizer.hpp:65) */
    uint32_t num_buckets;
    const char* tmp_dir;      /* bucket_<b>.bin written here */
    uint32_t host_threads;    /* inflate / parse / LZ4 threads (0 = all cores) */
    uint64_t chunk_bytes;     /* sequence bytes per device pass (0 = 8 GiB) */
    uint64_t* bucket_unc_bytes; /* out, num_buckets entries, may be NULL */
    uint32_t first_color;     /* color of files[0]: one rank's slice of a collection
                                 split by input file (0 for a whole build) */
} cdbg_phase1_args;

typedef struct cdbg_phase1_stats {
    uint64_t input_bytes;     /* on-disk bytes of the inputs */
    uint64_t seq_bytes;       /* sequence characters */
    uint64_t n_kmers;         /* k-mers in ACGT runs >= k (the throughput unit) */
    uint64_t n_supers;        /* super-k-mer occurrences */
    uint64_t n_records;       /* records written after dedup */
    uint64_t unc_bytes, comp_bytes;
    double seconds_total, seconds_device;
} cdbg_phase1_stats;

int cdbg_gpu_phase1(cdbg_engine* e, const cdbg_phase1_args* a, cdbg_phase1_stats* s);

/* Every super-k-mer occurrence of a batch in emission order, written to
 * dump_path as: u64 count, then per occurrence [u32 bucket][u8 flags]
 * [u32 color][u32 len][ceil(len/4) 2-bit packed bases].  Parity aid; the
 * layout matches the recording harness used to dump the reference's own
 * emit_super_kmers (bucket_ingester.hpp:36-127). */
int cdbg_gpu_dump_supers(cdbg_engine* e, const cdbg_seq_batch* b, uint32_t k, uint32_t m,
                         uint32_t num_buckets, const char* dump_path, uint64_t* n_supers);

/* Test aid (no counterpart in the reference): the device gzip decoder of the
 * device reader (gpu_inflate) on n gzip streams in host memory, inflated on
 * the device in one launch, one warp per stream.  outs[i] (host, out_caps[i]
 * bytes) receives stream i's bytes and out_lens[i] their count when
 * status[i] is 0; status 1 = more than out_caps[i] bytes, 2 = not a stream
 * the decoder accepts (the host reader's zlib then decides). */
int cdbg_gpu_gunzip(cdbg_engine* e, const uint8_t* const* streams, const uint64_t* lens, uint32_t n,
                    uint8_t* const* outs, const uint64_t* out_caps, uint64_t* out_lens, uint32_t* status);

/* Stable sort of n device (key, value) pairs by the full 64-bit key, in place
 * on the engine's stream: the sort phase 1 uses to order super-k-mers by
 * (bucket, hash) and phase 2 to group candidate color sets by hash (4 radix
 * passes over the top 32 key bits, then only the runs that tie there are
 * sorted on the rest).  Test aid, no counterpart in the reference. */
int cdbg_gpu_sort_pairs_u64(cdbg_engine* e, uint64_t* keys, uint32_t* vals, uint64_t n);

/* ---- phase 2 ------------------------------------------------------------ */

/* Called once per new color class in global cid order (the order the
 * reference's streaming_color_set_dict assigns ids when buckets are processed
 * in order by one thread).  `colors` is ascending. */
typedef void (*cdbg_class_cb)(void* ctx, const uint32_t* colors, uint64_t n);

typedef struct cdbg_phase2_args {
    const char* tmp_dir;         /* holds bucket_<b>.bin */
    uint32_t num_buckets;
    uint32_t k;
    uint32_t num_colors;
    const char* frag_path;       /* frag_unitigs.bin (unitig_spill.hpp:642-665 layout) */
    const char* color_sets_path; /* finalized .color_sets, or NULL */
    cdbg_class_cb on_class;      /* may be NULL */
    void* ctx;
    int32_t delete_consumed;     /* remove each bucket file once its fragments
                                    are written */
    uint32_t host_threads;
    uint64_t batch_occ;          /* k-mer occurrences per device batch (0 = auto) */
    uint64_t pass_bytes;         /* uncompressed bucket bytes read per pass:
                                    buckets are processed in consecutive ranges
                                    of at most this size (a larger bucket is a
                                    range of its own), the next range read on
                                    host threads while the device processes
                                    this one (0 = from free device memory) */
} cdbg_phase2_args;

typedef struct cdbg_phase2_stats {
    uint64_t n_records;
    uint64_t n_kmers;            /* k-mer occurrences rolled (reference "k-mers rolled") */
    uint64_t n_distinct;         /* distinct (bucket, canonical k-mer) nodes */
    uint64_t n_fragments;        /* frag_unitig_writer::count() */
    uint64_t total_seq_bytes;    /* frag_unitig_writer::total_seq_bytes() */
    uint64_t n_color_sets;       /* streaming_color_set_dict::size() */
    uint64_t total_integers;     /* sum of class sizes */
    uint64_t color_bits;         /* encoded bits of all classes */
    double seconds_total, seconds_device;
    uint64_t n_passes;           /* bucket ranges processed */
} cdbg_phase2_stats;

int cdbg_gpu_phase2(cdbg_engine* e, const cdbg_phase2_args* a, cdbg_phase2_stats* s);

/* ---- whole path in memory ---------------------------------------------- */

typedef struct cdbg_build_params {
    uint32_t k, m, num_buckets, num_colors;
    uint64_t batch_occ;          /* 0 = auto */
    int32_t outputs_to_host;     /* 1 = copy frag bytes and color-set words to host */
    /* Build only buckets [bucket_lo, bucket_hi) (both 0 = all): one rank's
     * share of a build split by bucket range, whose outputs
     * cdbg_merge_shards combines.  The rank still reads the whole input. */
    uint32_t bucket_lo, bucket_hi;
} cdbg_build_params;

typedef struct cdbg_build_result {
    /* Owned by the engine, valid until its next call.  Host pointers when
     * outputs_to_host = 1, else device pointers. */
    const uint8_t* frag_bytes;   /* frag_unitigs.bin contents */
    uint64_t frag_nbytes;
    const uint64_t* class_words; /* .color_sets bit-vector words */
    uint64_t class_bits;
    const uint64_t* class_offsets; /* bit offset of each class */
    uint64_t n_color_sets;
    uint64_t total_integers;
    uint64_t n_kmers, n_supers, n_records, n_occ, n_distinct, n_fragments, total_seq_bytes;
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t n_bases;            /* bases in ACGT runs >= k */
    double ms_phase1, ms_phase2, ms_total; /* device time (CUDA events) */
    double ms_outputs;           /* cdbg_gpu_build_files: wall time after phase 2
                                    (output copies and file writes left) */
    double ms_seed;              /* cdbg_gpu_build_files with stitch_dir: wall time
                                    of the round-0 seed (included in ms_outputs) */
    uint64_t seed_routed, seed_closed_unitigs;
} cdbg_build_result;

int cdbg_gpu_build(cdbg_engine* e, const cdbg_seq_batch* b, const cdbg_build_params* p,
                   cdbg_build_result* r);

/* The in-memory build from files, end to end: gzip/plain FASTA/FASTQ files
 * (file i = color i) in, frag_unitigs.bin and a finalized .color_sets out --
 * the inputs and outputs of the reference's phase 1 + phase 2 (builder.hpp:
 * 180-271) without its bucket files.  Host threads inflate and parse the
 * files in groups while the device already runs phase 1 on the groups read
 * before; phase 2 follows in HBM; the Elias-Fano finalize of the class
 * offsets (streaming_color_set_dict.hpp:221-294) runs on the device; the
 * outputs are written with parallel writes.  With both paths NULL the
 * outputs stay in host memory (the result's pointers, as cdbg_gpu_build with
 * outputs_to_host = 1).  r->ms_total is the call's wall time here. */
typedef struct cdbg_build_files_args {
    const char* const* files;
    uint32_t num_files;
    uint32_t k, m, num_buckets;    /* m = 0: compute_best_m(k) */
    uint32_t host_threads;         /* 0 = all cores */
    uint64_t batch_occ;            /* 0 = auto */
    const char* frag_path;         /* may be NULL */
    const char* color_sets_path;   /* may be NULL */
    /* Round 0 of the stitch from the fragments while they are in HBM: what
     * cdbg_gpu_stitch_seed writes from a frag file, without the file.  With
     * stitch_dir set, the round-0 files go there and the closed unitigs to
     * stitch_closed_path (NULL: stitch_dir/stitch_r0_closed.bin); frag_path may
     * then be NULL (no frag file, and no fragments in the result). */
    const char* stitch_dir;
    const char* stitch_closed_path;
    uint32_t stitch_buckets;       /* round-store buckets; 0 = 1024 */
    uint32_t stitch_kmer_bits;     /* as cdbg_seed_args.kmer_bits */
} cdbg_build_files_args;

int cdbg_gpu_build_files(cdbg_engine* e, const cdbg_build_files_args* a, cdbg_build_result* r);

/* ---- builds split across ranks ----------------------------------------- */

/* Merge the outputs of a build split by bucket range (cdbg_build_params
 * bucket_lo/bucket_hi), shards given in bucket order, into the outputs of the
 * whole build: the fragments back to back with their color-set ids rewritten
 * to the whole build's ids, and the color-set bit vector and offsets of the
 * whole build (its classes numbered by first appearance over all buckets, as
 * one build numbers them).  Host only (no GPU needed).  No counterpart in
 * the reference, which builds in one process.  The result's buffers belong to
 * the library until cdbg_merged_free; errors via cdbg_merge_last_error(). */
typedef struct cdbg_merged {
    const uint8_t* frag_bytes;
    uint64_t frag_nbytes;
    const uint64_t* class_words;
    uint64_t class_bits;
    const uint64_t* class_offsets;
    uint64_t n_color_sets;
    void* handle;
} cdbg_merged;

int cdbg_merge_shards(uint32_t num_shards, const uint8_t* const* frag, const uint64_t* frag_nbytes,
                      const uint64_t* const* class_words, const uint64_t* class_bits,
                      const uint64_t* const* class_offsets, const uint64_t* n_classes, cdbg_merged* out);
void cdbg_merged_free(cdbg_merged* m);
const char* cdbg_merge_last_error(void);

/* ---- round 0 of the phase-3 stitch ------------------------------------- */

/* The frag-file seed of the stitch: every fragment of a frag_unitigs.bin
 * (unitig_spill.hpp:491-522 records) becomes a round-0 tig in the round-store
 * bucket of the canonical boundary k-mer it presents, or, when it has no open
 * end, the monochromatic unitigs it splits into (stitch_extmem.hpp:930-944).
 * Outputs:
 *   round_dir/stitch_r0_b<b>.bin  the round store's round-0 files, byte for
 *       byte as a one-thread reference seed writes them (tigs of a bucket in
 *       fragment order, ext_tig_serialize layout, 4 MiB LZ4 frames, end
 *       mark); earlier round-0 files of buckets [0, num_buckets) there are
 *       removed first.  The reference's rounds continue from them:
 *       round_store_file store(round_dir, num_buckets); store.advance();
 *       ext_run_rounds(store, k, num_buckets, sink, done, T).
 *   the closed fragments' unitigs as frag records, fragment order: what the
 *       reference passes to `sink` during the seed (and counts in `done`),
 *       written to closed_path, or, with closed_path NULL, left in host
 *       memory owned by the engine (s->closed, valid until its next call).
 * With many threads the reference appends a bucket's tigs in the order its
 * workers finish; the rounds do not depend on that order (each tig's random
 * state comes from its bases). */
typedef struct cdbg_seed_args {
    const uint8_t* frags;       /* frag_unitigs.bin contents, host memory */
    uint64_t frag_nbytes;
    uint32_t k;
    uint32_t num_buckets;       /* round-store buckets; 0 = 1024 */
    uint32_t kmer_bits;         /* width of the reference build's kmer_int_t: 64, 128
                                   (CDBG_LARGE_K), or 0 = 64 for k <= 31, else 128 */
    uint32_t host_threads;      /* 0 = all cores */
    uint64_t chunk_bytes;       /* fragment bytes per device pass; 0 = auto */
    const char* round_dir;
    const char* closed_path;    /* may be NULL */
} cdbg_seed_args;

typedef struct cdbg_seed_stats {
    uint64_t fragments, routed, closed_fragments, closed_unitigs;
    uint64_t routed_frag_bytes; /* frag record bytes of the open fragments */
    uint64_t round0_bytes;      /* serialized tigs (uncompressed) */
    uint64_t round0_file_bytes; /* the round-0 files on disk */
    const uint8_t* closed;      /* closed unitigs when closed_path is NULL */
    uint64_t closed_nbytes;
    uint64_t n_passes;
    double ms_scan;             /* host: record offsets */
    double ms_device;           /* device time of the seed kernels (CUDA events) */
    double ms_files;            /* host: round-0 frames compressed and written, closed unitigs written */
    double ms_total;            /* wall time of the call */
} cdbg_seed_stats;

int cdbg_gpu_stitch_seed(cdbg_engine* e, const cdbg_seed_args* a, cdbg_seed_stats* s);

/* Byte offsets of the records of a frag_unitigs.bin buffer, found by several
 * host threads (each guesses a record start in its share of the buffer and
 * follows the records from there; the shares are joined where they meet the
 * records followed from the buffer's start, so the result is exact).  Writes
 * n_records + 1 offsets (the last = frag_nbytes) when cap allows.  Host only;
 * fails on a record that runs past the end. */
int cdbg_frag_record_offsets(const uint8_t* frags, uint64_t frag_nbytes, uint32_t host_threads, uint64_t* offsets,
                             uint64_t cap, uint64_t* n_records);

/* Phase 1 split by input file: rank r runs phase 1 on its own consecutive
 * slice of the input files (colors = global file indices) and sends each
 * bucket's records to the rank that owns the bucket.  This merges, for the
 * owner's buckets [b_lo, b_hi), the records all ranks made (source s's bucket
 * b_lo + i is src[s][src_off[s][i] .. src_off[s][i + 1]), decompressed bucket
 * file bytes, sources in file order) into the records one phase 1 over all
 * the files makes: the super-k-mers stably ordered by their key, equal
 * neighbours merged with flags AND-ed and colors united.  num_buckets is the
 * whole build's B.  Host only; the result's buffers belong to the library
 * until cdbg_merged_records_free; errors via cdbg_merge_last_error().  No
 * counterpart in the reference, which builds in one process. */
typedef struct cdbg_merged_records {
    const uint8_t* bytes;        /* the records of the buckets back to back */
    uint64_t nbytes;
    const uint64_t* bucket_off;  /* b_hi - b_lo + 1 offsets into bytes */
    void* handle;
} cdbg_merged_records;

int cdbg_merge_bucket_records(uint32_t num_sources, const uint8_t* const* src, const uint64_t* const* src_off,
                              uint32_t num_buckets, uint32_t b_lo, uint32_t b_hi, cdbg_merged_records* out);
void cdbg_merged_records_free(cdbg_merged_records* m);

/* Color-set interning across ranks (hash-partitioned, instead of merging all
 * shards on one rank).  cdbg_class_strings: each of a shard's n classes (bits
 * [offsets[c], offsets[c + 1]) of words, the last ending at class_bits)
 * re-aligned to bit 0 in whole words, strings[string_off[c] ..
 * string_off[c + 1]) (strings_cap >= class_bits / 64 + n words), and a 64-bit
 * hash of it, hashes[c] (the owner rank is hash % ranks).
 * cdbg_frag_remap_classes: the color-set ids of frag records rewritten in
 * place through map[nmap] (foreign runs keep their marker).  Host only;
 * errors via cdbg_merge_last_error().  No counterpart in the reference. */
int cdbg_class_strings(const uint64_t* words, uint64_t class_bits, const uint64_t* offsets, uint64_t n,
                       uint64_t* hashes, uint64_t* strings, uint64_t strings_cap, uint64_t* string_off);
int cdbg_frag_remap_classes(uint8_t* frag, uint64_t n, const uint64_t* map, uint64_t nmap);

/* Serialized size of the bucket records of the engine's last cdbg_gpu_build
 * (the uncompressed bytes its bucket files would hold), counted on the device
 * outside the build.  Valid until the engine's next call. */
int cdbg_engine_record_bytes(cdbg_engine* e, uint64_t* bytes);

/* Autotuner: builds `b` repeatedly, searching the knobs of cdbg_tuning one at
 * a time (batch split threshold, minimizer tile, heavy-record threshold) and
 * keeping each value that lowers the best of `rounds` device times; the
 * engine keeps the winner.  Every trial's outputs are identical (the knobs
 * are performance-only).  No counterpart in the reference. */
int cdbg_engine_autotune(cdbg_engine* e, const cdbg_seq_batch* b, const cdbg_build_params* p,
                         uint32_t rounds, cdbg_tuning* best, double* best_ms);

/* Super-k-mers of pre-packed ACGT runs for callers that cannot allocate
 * device memory.  No counterpart in the reference (which has no GPU path).
 *
 * Who needs it: code that must not call cudaMalloc/cudaFree or anything that
 * allocates on the device -- for example inside a host application that owns
 * all device memory through its own pool or budget, or where allocation is
 * forbidden at that point.  Such a caller brings every input and output
 * array; this function allocates nothing.  Its working memory is a fixed
 * file-scope device array of about 24 MiB that every GPU loading this
 * library holds until the process exits.
 *
 * Inputs (device): `words` is a 2-bit stream (base i at bits 2*(i%32) of word
 * i/32, with at least two readable words after the last base), 16-byte
 * aligned; run r starts at base run_soff[r] (a multiple of 32) and has
 * run_len[r] >= k ACGT bases and color run_color[r].  A misaligned `words`
 * or a run shorter than k is rejected with an error before any tile runs.
 * Outputs (device, out_cap entries each): per
 * super-k-mer in emission order its stream start, length, color, flags
 * (bit 0 begin, 1 end, 2 owns-first, 3 owns-last) and bucket -- the same
 * super-k-mers cdbg_gpu_dump_supers reports.  *n_supers receives the count.
 * Runs on `stream` (a cudaStream_t as void*, NULL = default stream).
 *
 * Limit: at most 512 tiles per call, a run taking ceil((len - k + 2) / 2048)
 * tiles (so at most 512 runs and 1,048,576 (k-1)-mers); larger inputs are
 * rejected with an error, as is an output capacity below the count.
 * The first call on a device looks up the device address of the working
 * array (cudaGetSymbolAddress); make that first call before any stream
 * capture.  That address stays cached for the life of the process: after a
 * cudaDeviceReset it is stale, so do not call this function again in that
 * process.  Each call synchronizes `stream` to read counts back to the host.
 * All calls share the working array, which keeps the previous call's
 * contents: calls that overlap on the GPU (other streams or host threads)
 * race and must be serialized by the caller.  Errors are reported through
 * cdbg_last_error(). */
int cdbg_gpu_supers_noalloc(const uint64_t* words, const uint64_t* run_soff, const uint32_t* run_len,
                            const uint32_t* run_color, uint32_t num_runs, uint32_t k, uint32_t m,
                            uint32_t num_buckets, uint64_t* out_start, uint32_t* out_len,
                            uint32_t* out_color, uint32_t* out_flags, uint32_t* out_bucket,
                            uint64_t out_cap, uint64_t* n_supers, void* stream);

/* ---- build server (continuous batching) -------------------------------- */

/* Many independent builds on one GPU, accepted at any time.  No counterpart in
 * the reference (one build per process).  `slots` engines run admitted
 * requests concurrently, each on its own stream; a request is admitted when a
 * slot is free and its device-memory estimate (bytes_per_base * input bases +
 * floor_bytes) fits in what is left of hbm_budget -- or, when nothing runs, at
 * once with the whole budget.  Requests start in arrival order.  Every
 * request's outputs are those of the same build run alone. */
typedef struct cdbg_server cdbg_server;

typedef struct cdbg_server_params {
    int device;
    uint32_t slots;              /* concurrent builds (0 = 1) */
    uint64_t hbm_budget;         /* device bytes for all admitted builds */
    double bytes_per_base;       /* memory model (0 = 24) */
    uint64_t floor_bytes;        /* memory model floor (0 = 2 GiB) */
} cdbg_server_params;

typedef struct cdbg_request_result {
    int32_t status;              /* 0, or < 0 with `error` set */
    const char* error;
    /* owned by the server until cdbg_server_release */
    const uint8_t* frag_bytes;   /* frag_unitigs.bin contents */
    uint64_t frag_nbytes;
    const uint64_t* class_words; /* .color_sets bit-vector words */
    uint64_t class_bits;
    const uint64_t* class_offsets;
    uint64_t n_color_sets;
    uint64_t total_integers, n_kmers, n_distinct, n_fragments;
    uint64_t need_bytes, grant_bytes;   /* estimate and memory granted */
    double t_submit, t_start, t_done;   /* seconds on the server's clock */
    double ms_device;                   /* device time of the build */
} cdbg_request_result;

typedef struct cdbg_server_stats_t {
    uint64_t completed, failed, waiting;
    uint32_t running, peak_running;
    uint64_t reserved_bytes, peak_reserved_bytes;
    double clock_s;
} cdbg_server_stats_t;

int cdbg_server_create(const cdbg_server_params* p, cdbg_server** out);
/* The batch's host buffers must stay valid until the request is done. */
int cdbg_server_submit(cdbg_server* s, const cdbg_seq_batch* host_batch, const cdbg_build_params* p,
                       uint64_t* request_id);
/* Blocks until the request is done. */
int cdbg_server_wait(cdbg_server* s, uint64_t request_id, cdbg_request_result* out);
int cdbg_server_release(cdbg_server* s, uint64_t request_id);
int cdbg_server_stats(cdbg_server* s, cdbg_server_stats_t* out);
/* Finishes every submitted request, then frees the engines. */
void cdbg_server_destroy(cdbg_server* s);
const char* cdbg_server_last_error(void);

/* Copy `bytes` from a device pointer returned by cdbg_gpu_build
 * (outputs_to_host = 0) into host memory, on the engine's stream. */
int cdbg_engine_copy_out(cdbg_engine* e, const void* device_src, void* host_dst, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif
