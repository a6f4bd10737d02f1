// Engine state shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "arena.cuh"
#include "common.cuh"

struct cdbg_engine {
    int device = 0;
    cudaStream_t st = nullptr;      // stream all work runs on
    cudaStream_t own_st = nullptr;  // the engine's own stream
    cdbg::kernel_profiler prof;
    cdbg::dev_arena A;   // per-stage scratch
    cdbg::dev_arena P;   // phase-1 outputs kept through phase 2 (in-memory build)
    // device-resident outputs of the last cdbg_gpu_build (outputs_to_host = 0)
    cdbg::dvec<uint8_t> out_frag;
    cdbg::dvec<uint64_t> out_words, out_offsets;
    uint32_t* d_err = nullptr;  // device error word (outside the arena)
    // outputs of the last cdbg_gpu_build (host copies)
    std::vector<uint8_t> h_frag;
    std::vector<uint64_t> h_words, h_offsets;
};

namespace cdbg {

// Throws when the device error word is set; clears it.
void check_device_error(cdbg_engine* e, char const* stage);

}  // namespace cdbg
