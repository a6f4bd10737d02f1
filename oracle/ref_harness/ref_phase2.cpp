// Phase-2 reference runner: the reference's own public process_buckets
// (phase2_bucket_process/bucket_walker.hpp:608) over an existing directory of
// bucket files (bucket_<b>.bin, LZ4-framed super-k-mer records), with the
// reference's frag_unitig_writer (unitig_spill.hpp:445) and
// streaming_color_set_dict (streaming_color_set_dict.hpp:86) as sinks, then
// finalize() of the color sets as phase 4 would do (builder.hpp:424).
//
//   ref_phase2 <bucket_dir> <num_buckets> <k> <num_colors> <threads> <out_dir>
//
// Writes <out_dir>/frag_unitigs.bin and <out_dir>/out.color_sets and prints
// one line: fragments, total_seq_bytes, num_color_sets, seconds.
#include <chrono>
#include <cstdio>
#include <filesystem>
#include <iostream>
#include <mutex>
#include <string>

#include "phase2_bucket_process/bucket_walker.hpp"
#include "phase2_bucket_process/streaming_color_set_dict.hpp"
#include "phase2_bucket_process/unitig_spill.hpp"

namespace fs = std::filesystem;

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s bucket_dir num_buckets k num_colors threads out_dir\n",
                     argv[0]);
        return 2;
    }
    const std::string in_dir = argv[1];
    const uint32_t B = (uint32_t)std::stoul(argv[2]);
    const uint32_t k = (uint32_t)std::stoul(argv[3]);
    const uint64_t C = std::stoull(argv[4]);
    const uint32_t T = (uint32_t)std::stoul(argv[5]);
    const std::string out_dir = argv[6];
    fs::create_directories(out_dir);
    const std::string work = out_dir + "/buckets";
    // The writer truncates its bucket files on construction; close it at once
    // (EOF markers only) and then copy the bucket files under test over them.
    cdbg::bucket_writer writer(work, B);
    writer.close();
    writer.release_compactors();
    for (uint32_t b = 0; b < B; ++b) {
        const std::string src = in_dir + "/bucket_" + std::to_string(b) + ".bin";
        if (fs::exists(src))
            fs::copy_file(src, writer.bucket_path(b), fs::copy_options::overwrite_existing);
    }
    cdbg::frag_unitig_writer frag_sink(out_dir + "/frag_unitigs.bin");
    cdbg::streaming_color_set_dict global_dict((uint32_t)C, out_dir + "/out.color_sets");
    std::mutex mu;
    auto t0 = std::chrono::steady_clock::now();
    cdbg::process_buckets(writer, k, C, T, frag_sink, global_dict, mu, nullptr, 0, false);
    auto t1 = std::chrono::steady_clock::now();
    const uint64_t ncs = global_dict.size();
    global_dict.release_index();
    frag_sink.close_for_writing();
    global_dict.finalize();
    std::printf("fragments=%llu total_seq_bytes=%llu num_color_sets=%llu seconds=%.6f\n",
                (unsigned long long)frag_sink.count(),
                (unsigned long long)frag_sink.total_seq_bytes(), (unsigned long long)ncs,
                std::chrono::duration<double>(t1 - t0).count());
    fs::remove_all(work);
    return 0;
}
