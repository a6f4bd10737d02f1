// Stitch round-0 runner: the reference's own frag-file seed
// (phase3_stitch/stitch_extmem.hpp:1013-1099, detail::ext_seed_round0_raw_par)
// over a frag_unitigs.bin, with the round store and sink that
// stitch_unitigs_extmem_file_streaming (:1120-1129) and builder.hpp:369-391
// give it: a round_store_file in <out_dir> and, for the closed fragments'
// unitigs, a frag_unitig_writer (unitig_spill.hpp:445-482) to
// <out_dir>/closed.bin.  Nothing after the seed runs, so the round-0 files
// <out_dir>/stitch_r0_b<b>.bin stay on disk.
//
//   ref_seed <frag_file> <k> <num_buckets> <threads> <out_dir>
//
// With threads = 1 the seed is serial and its files are deterministic.
// Prints one line: fragments, closed unitigs, seconds of the seed.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <filesystem>
#include <functional>
#include <string>

#include "phase2_bucket_process/unitig_spill.hpp"
#include "phase3_stitch/stitch_extmem.hpp"

namespace fs = std::filesystem;

int main(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s frag_file k num_buckets threads out_dir\n", argv[0]);
        return 2;
    }
    try {
        const std::string frag_path = argv[1];
        const uint32_t k = (uint32_t)std::stoul(argv[2]);
        const uint32_t B = (uint32_t)std::stoul(argv[3]);
        const uint32_t T = (uint32_t)std::stoul(argv[4]);
        const std::string out = argv[5];
        fs::create_directories(out);
        uint64_t n_frags = 0;
        auto for_each_raw = [&](auto&& fn) {
            cdbg::frag_unitig_block_reader rd(frag_path);
            uint8_t const* rec;
            uint32_t len;
            while (rd.next_raw(rec, len)) {
                ++n_frags;
                fn(rec, len);
            }
        };
        cdbg::frag_unitig_writer closed(out + "/closed.bin");
        std::atomic<uint64_t> done{0};
        cdbg::detail::round_store_file store(out, B);
        const auto t0 = std::chrono::steady_clock::now();
        cdbg::detail::ext_seed_round0_raw_par(for_each_raw, cdbg::frag_record_parse, k, store, std::ref(closed),
                                              &done, T);
        const auto t1 = std::chrono::steady_clock::now();
        closed.close_for_writing();
        std::printf("fragments=%llu closed_unitigs=%llu seconds=%.6f\n", (unsigned long long)n_frags,
                    (unsigned long long)done.load(), std::chrono::duration<double>(t1 - t0).count());
    } catch (std::exception const& e) {
        std::fprintf(stderr, "ref_seed: %s\n", e.what());
        return 1;
    }
    return 0;
}
