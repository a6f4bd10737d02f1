/* Seeded synthetic pangenome generator (benchmark / test workloads).
 *
 * No counterpart in the reference, which ships only two real data sets
 * (test_data/salmonella_10, test_data/se-50.tar.gz).  The parameters express
 * the genome shapes of the five benchmark workloads: small 10-genome set,
 * 1000-genome pangenome, 500-genome large-k set with repeats, 2000-genome
 * skewed set with low-complexity content, and per-request serving sets. */
#ifndef CDBG_SYNTH_H
#define CDBG_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cdbg_synth_params {
    uint64_t seed;
    double len_min, len_max;        /* genome length (bp); log-uniform when different */
    double div_min, div_max;        /* per-genome SNP rate, uniform */
    uint32_t indels;                /* indels of 1-50 bp per genome */
    uint32_t mobile_pool;           /* shared mobile elements; one inserted per genome */
    uint32_t mobile_min, mobile_max;
    uint32_t repeat_pool;           /* shared 1-5 kbp repeats */
    uint32_t repeats_per_genome;
    uint32_t contigs_min, contigs_max;
    uint32_t contigs_log;           /* 1 = log-uniform contig count */
    double tandem_frac;             /* tandem-repeat content of the ancestor */
    double lowcomp_frac;            /* homopolymer / dinucleotide content of the ancestor */
    uint32_t lowercase_runs;        /* 1 = lower-case a few 50-bp stretches */
    uint32_t n_runs;                /* 1 = insert a few short N runs */
} cdbg_synth_params;

/* One genome, contigs back to back in `out`; returns total bytes, or the
 * size alone when out == NULL, -1 when a capacity is too small. */
int64_t cdbg_synth_genome(const cdbg_synth_params* p, uint32_t genome, char* out, uint64_t cap,
                          uint64_t* contig_lens, uint32_t contig_cap, uint32_t* num_contigs);

/* Genomes [g0, g1) back to back, generated by `threads` threads. */
int64_t cdbg_synth_collection(const cdbg_synth_params* p, uint32_t g0, uint32_t g1,
                              uint32_t threads, char* out, uint64_t cap, uint64_t* contig_lens,
                              uint64_t contig_cap, uint32_t* contigs_per_genome,
                              uint64_t* total_contigs);

/* Write genomes [g0, g1) as <out_dir>/g<i>.fa (or .fa.gz when gzip_level > 0)
 * and a filenames list, line i = genome g0 + i. Returns 0 on success. */
int cdbg_synth_write_fasta(const cdbg_synth_params* p, uint32_t g0, uint32_t g1,
                           const char* out_dir, int gzip_level, uint32_t threads,
                           const char* filelist_path);

#ifdef __cplusplus
}
#endif

#endif
