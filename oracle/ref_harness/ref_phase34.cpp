// Phase-3/4 runner: the reference's own stitch (phase3_stitch/stitch_extmem.hpp:1120)
// and emit (phase4_emit/emit.hpp:93,177) over phase-2 artifacts produced by
// another implementation -- a frag_unitigs.bin and the list of color classes in
// global-id order.  This is the call sequence builder.hpp:297-440 runs after
// process_buckets, with the phase-2 outputs read from files instead of the
// in-process frag_unitig_writer / streaming_color_set_dict.
//
//   ref_phase34 <frag_file> <classes_file> <num_colors> <k> <threads> <out_basename> <tmp_dir>
//               [<seed_closed_file>]
//
// With seed_closed_file, round 0 of the stitch comes from another
// implementation: tmp_dir already holds the round-0 files stitch_r0_b<b>.bin
// of 1024 round-store buckets, and seed_closed_file the closed fragments'
// unitigs (frag records) that the seed would have passed to the sink.  They
// go to the sink, the round store is advanced past round 0 and the
// reference's doubling rounds (stitch_extmem.hpp:625, ext_run_rounds) run as
// stitch_unitigs_extmem_file_streaming runs them after its seed (:1127-1128).
//
// classes_file: u64 count, then per class u32 n followed by n ascending u32
// colors.  Every class is interned into a streaming_color_set_dict in file
// order (ids 0, 1, ... as phase 2 assigned them), which writes
// <out_basename>.color_sets exactly as process_buckets' merge would.
//
// Writes <out_basename>.fa/.u2c/.color_sets/.metadata.txt and prints one line
// of counts.  Test infrastructure: proves the GPU phase-2 artifacts drive the
// unchanged reference phases 3 and 4.
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "phase2_bucket_process/streaming_color_set_dict.hpp"
#include "phase2_bucket_process/unitig_spill.hpp"
#include "phase3_stitch/stitch_extmem.hpp"
#include "phase4_emit/emit.hpp"

namespace fs = std::filesystem;

static std::vector<std::vector<uint32_t>> read_classes(std::string const& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    uint64_t n = 0;
    if (std::fread(&n, 8, 1, f) != 1) throw std::runtime_error("short classes file");
    std::vector<std::vector<uint32_t>> out(n);
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t m = 0;
        if (std::fread(&m, 4, 1, f) != 1) throw std::runtime_error("short classes file");
        out[i].resize(m);
        if (m && std::fread(out[i].data(), 4, m, f) != m) throw std::runtime_error("short classes file");
    }
    std::fclose(f);
    return out;
}

int main(int argc, char** argv) {
    if (argc != 8 && argc != 9) {
        std::fprintf(stderr,
                     "usage: %s frag_file classes_file num_colors k threads out_basename tmp_dir [seed_closed_file]\n",
                     argv[0]);
        return 2;
    }
    try {
        const std::string frag_path = argv[1];
        const std::string classes_path = argv[2];
        const uint64_t C = std::stoull(argv[3]);
        const uint32_t k = (uint32_t)std::stoul(argv[4]);
        const uint32_t T = (uint32_t)std::stoul(argv[5]);
        const std::string out = argv[6];
        const std::string tmp_dir = argv[7];
        fs::create_directories(tmp_dir);

        // phase-2 color classes -> the streaming dict (writes <out>.color_sets)
        cdbg::streaming_color_set_dict global_dict((uint32_t)C, out + ".color_sets");
        for (auto& cl : read_classes(classes_path)) global_dict.intern(std::move(cl));
        const uint64_t num_color_sets = global_dict.size();
        global_dict.release_index();

        // the frag writer's counters (count(), total_seq_bytes()), from the file
        uint64_t n_frags = 0, total_frag_seq_bytes = 0;
        {
            cdbg::frag_unitig_block_reader rd(frag_path);
            uint8_t const* rec;
            uint32_t len;
            uint8_t fl;
            std::vector<cdbg::color_run> runs;
            std::string seq;
            while (rd.next_raw(rec, len)) {
                cdbg::frag_record_parse(rec, len, fl, runs, seq);
                ++n_frags;
                total_frag_seq_bytes += seq.size();
            }
        }

        // Bucket counts the builder picks without -g: min(num_color_sets, 64)
        // unitig buckets (builder.hpp:766-778) and 1024 stitch buckets
        // (builder.hpp:808-822).
        const uint64_t unitig_buckets = num_color_sets == 0 ? 1 : std::min<uint64_t>(num_color_sets, 64);
        cdbg::unitig_bucket_writer uwriter(tmp_dir, num_color_sets, (uint32_t)unitig_buckets, SIZE_MAX);
        auto for_each_raw = [&](auto&& fn) {
            cdbg::frag_unitig_block_reader rd(frag_path);
            uint8_t const* rec;
            uint32_t len;
            while (rd.next_raw(rec, len)) fn(rec, len);
        };
        if (argc == 9) {
            cdbg::frag_unitig_block_reader rd(argv[8]);
            uint8_t const* rec;
            uint32_t len;
            while (rd.next_raw(rec, len)) {
                cdbg::stitchable_unitig u;
                cdbg::frag_record_parse(rec, len, u.open_flags, u.runs, u.seq);
                uwriter(std::move(u));
            }
            cdbg::detail::round_store_file store(tmp_dir, 1024);
            store.advance();
            cdbg::detail::ext_run_rounds(store, k, 1024, std::ref(uwriter), nullptr, T);
        } else {
            cdbg::stitch_unitigs_extmem_file_streaming(for_each_raw, cdbg::frag_record_parse, k, tmp_dir,
                                                       std::ref(uwriter), 1024, nullptr, T);
        }
        const uint64_t num_unitigs = uwriter.total_unitigs();
        const uint64_t num_kmers = uwriter.total_seq_bytes() - num_unitigs * (uint64_t)(k - 1);
        cdbg::emit_fasta(uwriter, out, num_unitigs, 0.0);
        cdbg::emit_colors(global_dict);

        // metadata lines of builder.hpp:754-764
        std::ofstream md(out + ".metadata.txt");
        md << "k=" << k << "\n"
           << "num_kmers=" << num_kmers << "\n"
           << "num_colors=" << C << "\n"
           << "num_unitigs=" << num_unitigs << "\n"
           << "num_color_sets=" << num_color_sets << "\n";
        if (!md) throw std::runtime_error("failed writing metadata");
        std::printf("fragments=%llu frag_seq_bytes=%llu unitigs=%llu kmers=%llu color_sets=%llu\n",
                    (unsigned long long)n_frags, (unsigned long long)total_frag_seq_bytes,
                    (unsigned long long)num_unitigs, (unsigned long long)num_kmers,
                    (unsigned long long)num_color_sets);
    } catch (std::exception const& e) {
        std::fprintf(stderr, "ref_phase34: %s\n", e.what());
        return 1;
    }
    return 0;
}
