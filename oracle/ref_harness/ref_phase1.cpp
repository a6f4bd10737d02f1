// Phase-1 golden-vector generator: runs the reference's own
// detail::ingest_file_bucketed (phase1_bucket_write/bucket_ingester.hpp:129)
// -- and through it seq_reader, the ACGT scan, windowed_min and
// emit_super_kmers -- over a list of FASTA/FASTQ(.gz) files, file i = color i,
// and dumps every super-k-mer occurrence in emission order.
//
//   ref_phase1 <filenames.txt> <k> <m> <num_buckets> <out.bin>
//
// out.bin: u64 count, then per occurrence
//   [u32 bucket][u8 flags][u32 color][u32 len][ceil(len/4) bytes, 2-bit packed
//    LSB-first exactly like super_kmer.hpp:43 pack_2bit]
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "phase1_bucket_write/bucket_ingester.hpp"

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s filenames.txt k m num_buckets out.bin\n", argv[0]);
        return 2;
    }
    std::vector<std::string> files;
    {
        std::ifstream in(argv[1]);
        std::string line;
        while (std::getline(in, line))
            if (!line.empty()) files.push_back(line);
    }
    const uint32_t k = (uint32_t)std::stoul(argv[2]);
    uint32_t m = (uint32_t)std::stoul(argv[3]);
    if (m == 0) m = cdbg::compute_best_m(k);
    const uint32_t B = (uint32_t)std::stoul(argv[4]);
    cdbg::bucket_writer w;
    cdbg::per_thread_bucket_buffers sink(w);
    for (uint32_t i = 0; i < files.size(); ++i)
        cdbg::detail::ingest_file_bucketed(files[i], k, m, B, i, sink);
    auto const& v = cdbg::recorded_supers();
    std::FILE* f = std::fopen(argv[5], "wb");
    if (!f) return 1;
    uint64_t n = v.size();
    std::fwrite(&n, 8, 1, f);
    std::vector<uint8_t> packed;
    for (auto const& r : v) {
        std::fwrite(&r.bucket, 4, 1, f);
        std::fwrite(&r.flags, 1, 1, f);
        std::fwrite(&r.color, 4, 1, f);
        uint32_t len = (uint32_t)r.bases.size();
        std::fwrite(&len, 4, 1, f);
        packed.clear();
        cdbg::pack_2bit(r.bases.data(), len, packed);
        std::fwrite(packed.data(), 1, packed.size(), f);
    }
    std::fclose(f);
    std::printf("m=%u supers=%llu\n", m, (unsigned long long)n);
    return 0;
}
