// Phase 1 + phase 2 of the reference, exactly as its builder runs them, and
// nothing after: the CPU baseline of the benchmarks.
//
//   ref_phase12 <filenames_list> <k> <m|0> <num_buckets> <threads> <tmp_dir> <out_dir>
//
// The calls and their arguments follow builder.hpp:133-271: a bucket_writer
// with the builder's default flush/spill sizes (builder.hpp:524-525, 577-578),
// ingest_bucketed over the files (bucket_ingester.hpp:183), close() and
// release_compactors(), then process_buckets with the reference's
// frag_unitig_writer and streaming_color_set_dict as sinks
// (bucket_walker.hpp:607), deleting each bucket file once consumed as the
// builder does without --keep-tmp.  m = 0 means compute_best_m(k)
// (minimizer.hpp:65).  No -g budget.
//
// Prints the reference's own phase timers (the builder times ingest_bucketed
// as "bucket-write" and process_buckets as "bucket-process") and one summary
// line: seconds of the whole phase-1 + phase-2 span (close() included),
// fragments, distinct color sets.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <mutex>
#include <string>
#include <vector>

#include "phase1_bucket_write/bucket_ingester.hpp"
#include "phase1_bucket_write/minimizer.hpp"
#include "phase2_bucket_process/bucket_walker.hpp"
#include "phase2_bucket_process/streaming_color_set_dict.hpp"
#include "phase2_bucket_process/unitig_spill.hpp"

namespace fs = std::filesystem;

int main(int argc, char** argv) {
    if (argc != 8) {
        std::fprintf(stderr, "usage: %s filenames_list k m num_buckets threads tmp_dir out_dir\n", argv[0]);
        return 2;
    }
    std::vector<std::string> files;
    {
        std::ifstream in(argv[1]);
        if (!in) {
            std::fprintf(stderr, "cannot open %s\n", argv[1]);
            return 1;
        }
        std::string line;
        while (std::getline(in, line))
            if (!line.empty()) files.push_back(line);
    }
    const uint32_t k = (uint32_t)std::stoul(argv[2]);
    uint32_t m = (uint32_t)std::stoul(argv[3]);
    if (m == 0) m = cdbg::compute_best_m(k);
    const uint32_t B = (uint32_t)std::stoul(argv[4]);
    const uint32_t T = (uint32_t)std::stoul(argv[5]);
    const std::string tmp = argv[6], out = argv[7];
    fs::create_directories(tmp);
    fs::create_directories(out);
    const uint64_t C = files.size();

    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    cdbg::bucket_writer writer(tmp, B, 4 * 1024, 64 * 1024);
    ingest_bucketed(files, k, m, B, writer, T);
    const auto t1 = clk::now();
    writer.close();
    writer.release_compactors();
    cdbg::frag_unitig_writer frag_sink(tmp + "/frag_unitigs.bin");
    cdbg::streaming_color_set_dict global_dict((uint32_t)C, out + "/out.color_sets");
    std::mutex mu;
    std::atomic<uint64_t> done{0};
    const auto t2 = clk::now();
    cdbg::process_buckets(writer, k, C, T, frag_sink, global_dict, mu, &done, 0, true);
    const auto t3 = clk::now();
    auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    std::printf("[bucket-write] %.6f s\n[bucket-process] %.6f s\n", sec(t0, t1), sec(t2, t3));
    std::printf("phase12_seconds=%.6f fragments=%llu num_color_sets=%llu k=%u m=%u buckets=%u threads=%u\n",
                sec(t0, t3), (unsigned long long)frag_sink.count(), (unsigned long long)global_dict.size(), k, m,
                B, T);
    return 0;
}
