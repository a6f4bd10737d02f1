// Shared device/host helpers for the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace cdbg {

typedef unsigned __int128 u128;

extern std::atomic<uint64_t> g_launches;

// Message returned by cdbg_last_error() (thread-local).
void set_last_error(std::string const& msg);

// Per-kernel device time with CUDA events on the launching stream.  Enabled
// per engine call; a scope records an event before and after the launch it
// encloses, and resolve() folds the finished pairs into per-name totals.
struct kernel_profiler {
    struct pending {
        char const* name;
        cudaEvent_t a, b;
    };
    bool on = false;
    std::vector<pending> open;
    std::vector<cudaEvent_t> pool;
    std::map<std::string, std::pair<double, uint64_t>> totals;  // ms, launches
    std::map<std::string, double> bytes;  // algorithmic bytes declared at the launch sites
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void resolve() {
        for (auto& p : open) {
            float ms = 0;
            cudaEventSynchronize(p.b);
            cudaEventElapsedTime(&ms, p.a, p.b);
            auto& t = totals[p.name];
            t.first += ms;
            t.second += 1;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        open.clear();
    }
    ~kernel_profiler() {
        resolve();
        for (auto e : pool) cudaEventDestroy(e);
    }
};
extern thread_local kernel_profiler* g_prof;

struct prof_scope {
    kernel_profiler* p;
    cudaStream_t st;
    char const* name;
    cudaEvent_t a{};
    prof_scope(char const* n, cudaStream_t s, double alg_bytes = 0)
        : p(g_prof && g_prof->on ? g_prof : nullptr), st(s), name(n) {
        if (p) {
            a = p->get();
            cudaEventRecord(a, st);
            if (alg_bytes > 0) p->bytes[name] += alg_bytes;
        }
    }
    ~prof_scope() {
        if (p) {
            cudaEvent_t b = p->get();
            cudaEventRecord(b, st);
            p->open.push_back({name, a, b});
        }
    }
};
#define CDBG_PROF(name, st) ::cdbg::prof_scope cdbg_prof_scope_(name, st)
// Same, declaring the algorithmic bytes the launch reads and writes (the
// roofline numerator: data it must move, not probes or re-reads).
#define CDBG_PROF_BYTES(name, st, bytes) ::cdbg::prof_scope cdbg_prof_scope_(name, st, (double)(bytes))

#define CDBG_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) +    \
                                     " at " + __FILE__ + ":" + std::to_string(__LINE__));      \
    } while (0)

// Every kernel launch is followed by this check, which also counts launches
// (the count is exported through cdbg_launch_count()).
#define CDBG_CHECK_LAUNCH()                 \
    do {                                    \
        ::cdbg::g_launches.fetch_add(1);    \
        CDBG_CUDA(cudaGetLastError());      \
    } while (0)

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

// ---- small device -> host reads
// The host waits for a few bytes of device memory (a count, a flag, digit
// histograms).  With a mailbox installed for the calling thread (mapped pinned
// host memory, installed by the engine for the duration of each call), a
// one-block kernel stores the bytes into it over PCIe, and no copy engine is
// involved: a cudaMemcpyAsync would wait behind the large output copies that
// stream to the host on the engine's copy stream (tens of milliseconds each)
// and stall every batch.  Without a mailbox it is a cudaMemcpyAsync.
struct host_mailbox {
    void* h = nullptr;  // host address
    void* d = nullptr;  // device address of the same pages
    size_t bytes = 0;
};
extern thread_local host_mailbox* g_mailbox;
// Radix digit width of the sorts run by this host thread's current engine
// call (8 or 11 bits; a performance knob, cdbg_tuning.radix_bits).
extern thread_local int g_radix_bits;

namespace {
__global__ void k_mail_bytes(uint8_t const* __restrict__ src, uint8_t* __restrict__ dst, uint64_t n) {
    if (((uintptr_t)src & 7) == 0 && (n & 7) == 0) {
        for (uint64_t i = threadIdx.x; i < n / 8; i += blockDim.x)
            reinterpret_cast<uint64_t*>(dst)[i] = reinterpret_cast<uint64_t const*>(src)[i];
    } else {
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    }
}

inline void read_small(void* host_dst, void const* dev_src, size_t n, cudaStream_t st) {
    host_mailbox* mb = g_mailbox;
    if (mb && mb->h && n <= mb->bytes) {
        k_mail_bytes<<<1, 256, 0, st>>>(static_cast<uint8_t const*>(dev_src), static_cast<uint8_t*>(mb->d), n);
        CDBG_CHECK_LAUNCH();
        CDBG_CUDA(cudaStreamSynchronize(st));
        std::memcpy(host_dst, mb->h, n);
    } else {
        CDBG_CUDA(cudaMemcpyAsync(host_dst, dev_src, n, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
    }
}
}  // namespace

}  // namespace cdbg
