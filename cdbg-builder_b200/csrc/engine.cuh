// Engine state shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "cdbg_gpu.h"
#include "arena.cuh"
#include "common.cuh"
#include "phase1.cuh"
#include "phase2.cuh"

// Page-locked host buffer grown on demand and kept by the engine, so host
// copies of build outputs run at full PCIe speed without re-pinning per call.
struct pinned_buffer {
    void* p = nullptr;
    size_t cap = 0;
    pinned_buffer() = default;
    pinned_buffer(pinned_buffer const&) = delete;
    ~pinned_buffer() {
        if (p) cudaFreeHost(p);
    }
    void* ensure(size_t n) {
        if (n <= cap && p) return p;
        if (p) cudaFreeHost(p);
        p = nullptr;
        size_t c = n > 2 * cap ? n : 2 * cap;
        if (c == 0) c = 4096;
        CDBG_CUDA(cudaMallocHost(&p, c));
        cap = c;
        return p;
    }
};

struct cdbg_engine {
    int device = 0;
    cudaStream_t st = nullptr;      // stream all work runs on
    cudaStream_t own_st = nullptr;  // the engine's own stream
    cudaStream_t copy_st = nullptr; // device-to-host copies that overlap phase 2
    cudaEvent_t copy_ev = nullptr;
    cdbg::kernel_profiler prof;
    cdbg::dev_arena A;   // per-stage scratch
    cdbg::dev_arena P;   // phase-1 outputs kept through phase 2 (in-memory build)
    // class dictionary + device-resident outputs, reused across builds
    cdbg::phase2_state p2;
    uint32_t* d_err = nullptr;  // device error word (outside the arena)
    uint64_t mem_limit = 0;     // device memory cap of this engine (0 = none)
    cdbg_tuning tune{0, 4096, 64, 8, 0, 0, 8, 0};
    cdbg::record_set last_rs;  // records of the last in-memory build (in P)
    bool have_rs = false;
    // host copies of the last cdbg_gpu_build's outputs (outputs_to_host = 1)
    pinned_buffer h_frag, h_words, h_offsets;
    // inflated input sequences of cdbg_gpu_build_files, read while the
    // device works on the groups read before
    pinned_buffer h_in;
    // set by cdbg_gpu_build_files while it writes the fragment file: phase 2
    // streams each batch's fragments to h_frag and calls `fn` (when h_frag is
    // already large enough); `streamed` receives the bytes so queued
    struct frag_sink_hook {
        void (*fn)(void*, uint64_t, uint64_t) = nullptr;
        void* ctx = nullptr;
        uint64_t streamed = 0;
    } frag_sink;
    // decompressed bucket ranges of the drop-in phase 2 (one read while the
    // device processes the other)
    pinned_buffer h_bk[2];
    std::vector<uint8_t> h_closed;  // cdbg_gpu_stitch_seed: closed unitigs kept in memory
    pinned_buffer h_tigs, h_unitigs;  // stitch seed: tigs and closed unitigs on their way to the files
    bool keep_frag_offsets = false;   // the next build keeps its fragment record offsets in p2.frag_off
    pinned_buffer h_rec_off;  // cdbg_gpu_stitch_seed: record offsets, reused between calls
    std::vector<std::vector<uint64_t>> h_rec_parts;
    // mapped pinned page for the small reads the host waits on (counts, flags,
    // histograms): written by a kernel, so they never queue behind the output
    // copies on the copy engine
    cdbg::host_mailbox mailbox;
};

namespace cdbg {

// Throws when the device error word is set; clears it.
void check_device_error(cdbg_engine* e, char const* stage);

}  // namespace cdbg
