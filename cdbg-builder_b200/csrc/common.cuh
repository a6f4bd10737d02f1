// Shared device/host helpers for the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace cdbg {

typedef unsigned __int128 u128;

#define CDBG_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +    \
                                     " at " + __FILE__ + ":" + std::to_string(__LINE__));      \
    } while (0)

#define CDBG_CHECK_LAUNCH() CDBG_CUDA(cudaGetLastError())

// Device-side error words.  Kernels never trap: a bounded loop that runs out,
// a table that fills up or a size that overflows a field sets a code here and
// the host turns it into an error return after the stage's synchronize.
enum dev_error : uint32_t {
    ERR_NONE = 0,
    ERR_TABLE_FULL = 1,       // open-addressing probe limit reached
    ERR_FIELD_OVERFLOW = 2,   // a value did not fit its packed field
    ERR_BAD_RECORD = 3,       // malformed serialized record
    ERR_CAPACITY = 4,         // an output buffer sized from a bound overflowed
    ERR_CHAIN_LIMIT = 5,      // a chain walk exceeded its step bound
};

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t code) {
    if (err) atomicCAS(err, 0u, code);
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Read 64 bits of a 2-bit-packed base stream starting at base `pos`
// (base i at bits 2*(i%32) of word i/32).  `words` must have one readable
// word past the last base (streams are allocated with padding).
__device__ __forceinline__ uint64_t stream_bits64(uint64_t const* __restrict__ words, uint64_t pos) {
    const uint64_t w = pos >> 5;
    const uint32_t s = (uint32_t)(pos & 31) * 2;
    uint64_t lo = __ldg(words + w) >> s;
    if (s) lo |= __ldg(words + w + 1) << (64 - s);
    return lo;
}

}  // namespace cdbg
