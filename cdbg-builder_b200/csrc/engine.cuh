// Engine state shared by the C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "arena.cuh"
#include "common.cuh"

struct cdbg_engine {
    int device = 0;
    cudaStream_t st = nullptr;
    cdbg::dev_arena A;
    uint32_t* d_err = nullptr;  // device error word (outside the arena)
    // outputs of the last cdbg_gpu_build (host copies)
    std::vector<uint8_t> h_frag;
    std::vector<uint64_t> h_words, h_offsets;
    // device-resident outputs of the last build (arena memory)
    uint8_t* d_frag = nullptr;
    uint64_t* d_words = nullptr;
    uint64_t* d_offsets = nullptr;
};

namespace cdbg {

// Throws when the device error word is set; clears it.
void check_device_error(cdbg_engine* e, char const* stage);

}  // namespace cdbg
