// Device-wide primitives written for this project: exclusive scan and a
// stable LSD radix sort of (key, value) pairs, u32 or u64 keys.
//
// Radix sort: one fused histogram pass computes the digit histograms of every
// requested pass in a single read of the keys; passes whose digit is constant
// over all keys are skipped.  Each executed pass is upsweep (per-tile digit
// counts, digit-major) -> exclusive scan of the counts -> downsweep.  The
// downsweep ranks keys stably inside a tile with warp match-any (each warp owns
// a contiguous slice of the tile, so warp order is tile order), stages the tile
// in shared memory in digit order and writes each digit's run contiguously.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "arena.cuh"
#include "common.cuh"

namespace cdbg {
namespace prim {
// Internal linkage: every translation unit that sorts gets its own copy.
namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename U>
__device__ __forceinline__ U warp_inclusive_scan(U v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        U t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total in *total.
template <typename U, int THREADS>
__device__ __forceinline__ U block_exclusive_scan(U v, U* smem_warp, U& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = THREADS / 32;
    U inc = warp_inclusive_scan(v);
    if (lane == 31) smem_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        U w = lane < NW ? smem_warp[lane] : U(0);
        U wi = warp_inclusive_scan(w);
        if (lane < NW) smem_warp[lane] = wi - w;
        if (lane == NW - 1) smem_warp[NW] = wi;
    }
    __syncthreads();
    U r = smem_warp[warp] + inc - v;
    total = smem_warp[NW];
    __syncthreads();
    return r;
}

// Tile sums: thread t adds elements t, t + 256, ... of the tile (coalesced).
template <typename T, typename U>
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(T const* __restrict__ in, uint64_t n,
                                                            U* __restrict__ sums) {
    __shared__ U sw[SCAN_THREADS / 32 + 1];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    U s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const uint64_t j = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
        if (j < n) s += (U)in[j];
    }
    U tot;
    block_exclusive_scan<U, SCAN_THREADS>(s, sw, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Shared-memory index of tile element j, padded so that a thread reading its
// SCAN_ITEMS consecutive elements meets no bank conflict (4- and 8-byte types).
template <typename V>
__device__ __forceinline__ uint32_t scan_pad(uint32_t j) {
    return j + (j >> (sizeof(V) == 8 ? 4 : 5));
}

// Tile scan: coalesced loads and stores through shared memory; each thread
// scans SCAN_ITEMS consecutive elements.
template <typename T, typename U>
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_scan(T const* __restrict__ in, uint64_t n,
                                                            U const* __restrict__ offs,
                                                            U* __restrict__ out, U* total_out) {
    __shared__ U sw[SCAN_THREADS / 32 + 1];
    __shared__ T sin[SCAN_TILE + SCAN_TILE / 16];
    __shared__ U sout[SCAN_TILE + SCAN_TILE / 16];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const uint32_t j = (uint32_t)i * SCAN_THREADS + threadIdx.x;
        sin[scan_pad<T>(j)] = (base + j < n) ? in[base + j] : T(0);
    }
    __syncthreads();
    T v[SCAN_ITEMS];
    U s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = sin[scan_pad<T>(threadIdx.x * SCAN_ITEMS + i)];
        s += (U)v[i];
    }
    U tot;
    U p = block_exclusive_scan<U, SCAN_THREADS>(s, sw, tot);
    p += offs ? offs[blockIdx.x] : U(0);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        sout[scan_pad<U>(threadIdx.x * SCAN_ITEMS + i)] = p;
        p += (U)v[i];
    }
    if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_THREADS - 1) *total_out = p;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        const uint32_t j = (uint32_t)i * SCAN_THREADS + threadIdx.x;
        if (base + j < n) out[base + j] = sout[scan_pad<U>(j)];
    }
}

// out[i] = sum(in[0..i)), in place allowed (out == in when T == U).  When
// total_dev is given the grand total is written there (device memory).
template <typename T, typename U>
void exclusive_scan(T const* in, U* out, uint64_t n, dev_arena& A, cudaStream_t st,
                    U* total_dev = nullptr) {
    if (n == 0) {
        if (total_dev) CDBG_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(U), st));
        return;
    }
    const uint64_t tiles = ceil_div(n, SCAN_TILE);
    auto m = A.mark();
    U* offs = nullptr;
    if (tiles > 1) {
        U* sums = A.alloc<U>(tiles);
        {
            CDBG_PROF("k_tile_sums", st);
            k_tile_sums<T, U><<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, n, sums);
        }
        CDBG_CHECK_LAUNCH();
        exclusive_scan<U, U>(sums, sums, tiles, A, st, (U*)nullptr);
        offs = sums;
    }
    {
        CDBG_PROF("k_tile_scan", st);
        k_tile_scan<T, U><<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, n, offs, out, total_dev);
    }
    CDBG_CHECK_LAUNCH();
    A.release(m);
}

// ------------------------------------------------------------ ordered output
// Decoupled look-back for tiles that take their indices in launch order from
// an atomic counter.  One warp of the tile calls it (all 32 lanes, the same
// arguments): lane 0 publishes the tile's count `tot` in status[tile]; the
// warp reads its predecessors' status 32 at a time (lane l the l-th nearest),
// adds their counts back to the nearest published inclusive prefix, lane 0
// publishes the tile's own inclusive prefix, and every lane gets the
// exclusive one in `excl`.  status[] is zeroed before the launch.  A
// predecessor took its index earlier, so it is running or done; every wait is
// still bounded, and on a timeout the tile publishes what it has (so its
// successors never wait on it) and returns false.
constexpr unsigned long long LB_AGG = 1ull << 62, LB_INC = 2ull << 62, LB_VAL = (1ull << 62) - 1;
__device__ __forceinline__ bool lookback_exclusive(unsigned long long* status, uint64_t tile, uint64_t tot,
                                                   uint64_t& excl) {
    const int lane = threadIdx.x & 31;
    excl = 0;
    if (tile == 0) {
        if (lane == 0) atomicExch(&status[0], LB_INC | tot);
        return true;
    }
    if (lane == 0) atomicExch(&status[tile], LB_AGG | tot);
    bool ok = true;
    uint64_t sum = 0;
    for (uint64_t end = tile;;) {  // window: tiles end - 1 - lane
        unsigned long long v = LB_INC;  // before tile 0: an inclusive prefix of 0
        if (end >= (uint64_t)lane + 1) {
            const uint64_t j = end - 1 - lane;
            for (uint32_t spin = 0; spin < (1u << 24); ++spin) {
                v = *(volatile unsigned long long*)&status[j];
                if (v >> 62) break;
            }
        }
        if (!__all_sync(0xffffffffu, (v >> 62) != 0)) {
            ok = false;
            break;
        }
        const uint32_t inc = __ballot_sync(0xffffffffu, (v >> 62) == 2);
        const int stop = inc ? __ffs(inc) - 1 : 31;  // nearest inclusive lane
        uint64_t x = lane <= stop ? (v & LB_VAL) : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        sum += x;
        if (inc) break;
        end -= 32;
    }
    if (lane == 0) atomicExch(&status[tile], LB_INC | ((sum + tot) & LB_VAL));
    excl = sum;
    return ok;
}

// ------------------------------------------------------------------ radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 2048
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_WARPS = RS_THREADS / 32;

// Histograms of all passes [begin_bit, end_bit) in one read.  hist is
// npasses x 256 u64, zeroed by the caller.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_histograms(K const* __restrict__ keys,
                                                              uint64_t n, int begin_bit,
                                                              int npasses,
                                                              unsigned long long* hist) {
    __shared__ uint32_t h[8][RS_BINS];
    for (int i = threadIdx.x; i < 8 * RS_BINS; i += RS_THREADS) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * RS_THREADS;
    for (uint64_t i = (uint64_t)blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += stride) {
        const K k = keys[i];
        for (int p = 0; p < npasses; ++p)
            atomicAdd(&h[p][(k >> (begin_bit + p * RS_BITS)) & (RS_BINS - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * RS_BINS; i += RS_THREADS) {
        const uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(&hist[i], (unsigned long long)v);
    }
}

// counts[d * ntiles + tile] = number of keys of tile with digit d.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(K const* __restrict__ keys,
                                                           uint64_t n, int shift, uint32_t ntiles,
                                                           uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[RS_BINS];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint64_t idx = base + (uint64_t)i * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (RS_BINS - 1)], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS) k_rs_downsweep(K const* __restrict__ keys_in,
                                                             V const* __restrict__ vals_in,
                                                             K* __restrict__ keys_out,
                                                             V* __restrict__ vals_out, uint64_t n,
                                                             int shift, uint32_t ntiles,
                                                             uint64_t const* __restrict__ offs) {
    __shared__ K sk[RS_TILE];
    __shared__ V sv[RS_TILE];
    __shared__ uint32_t wcnt[RS_WARPS][RS_BINS];  // per-warp digit counts, then prefixes
    __shared__ uint32_t dstart[RS_BINS];          // tile-local start of each digit
    __shared__ uint64_t gbase[RS_BINS];           // global start of each digit for this tile
    __shared__ uint32_t sw[RS_THREADS / 32 + 1];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();

    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    const uint32_t tile_n = (uint32_t)((n - base) < (uint64_t)RS_TILE ? (n - base) : RS_TILE);
    // Warp w owns tile positions [w*256, (w+1)*256): rounds of 32 in order.
    K k[RS_ITEMS];
    V v[RS_ITEMS];
    uint32_t rk[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const uint32_t pos = (uint32_t)warp * (RS_ITEMS * 32) + (uint32_t)r * 32 + lane;
        const bool ok = pos < tile_n;
        k[r] = ok ? keys_in[base + pos] : ~K(0);
        v[r] = ok ? vals_in[base + pos] : V(0);
        const uint32_t d = ok ? (uint32_t)((k[r] >> shift) & (RS_BINS - 1)) : RS_BINS;  // sentinel
        const uint32_t active = __ballot_sync(0xffffffffu, ok);
        const uint32_t peers = __match_any_sync(0xffffffffu, d) & active;
        uint32_t old = 0;
        const int leader = peers ? __ffs(peers) - 1 : 0;
        if (ok && lane == leader) {
            old = wcnt[warp][d];
            wcnt[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rk[r] = ok ? old + __popc(peers & lanemask_lt()) : 0;
    }
    __syncthreads();
    // Per digit: exclusive prefix over warps, and the digit's tile total.
    {
        const int d = threadIdx.x;  // RS_THREADS == RS_BINS
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<uint32_t, RS_THREADS>(run, sw, tot);
        dstart[d] = ex;
        gbase[d] = offs[(uint64_t)d * ntiles + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const uint32_t pos = (uint32_t)warp * (RS_ITEMS * 32) + (uint32_t)r * 32 + lane;
        if (pos < tile_n) {
            const uint32_t d = (uint32_t)((k[r] >> shift) & (RS_BINS - 1));
            const uint32_t lp = dstart[d] + wcnt[warp][d] + rk[r];
            sk[lp] = k[r];
            sv[lp] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < tile_n; p += RS_THREADS) {
        const K key = sk[p];
        const uint32_t d = (uint32_t)((key >> shift) & (RS_BINS - 1));
        const uint64_t dst = gbase[d] + (p - dstart[d]);
        keys_out[dst] = key;
        vals_out[dst] = sv[p];
    }
}

// Stable sort of (keys, vals) by key bits [begin_bit, end_bit).  Results end
// in (keys, vals); the arena provides the ping-pong buffers.  Needs a host
// synchronize (to read the digit histograms); returns the number of passes run.
template <typename V, typename K = uint64_t>
int radix_sort_pairs(K* keys, V* vals, uint64_t n, int begin_bit, int end_bit,
                     dev_arena& A, cudaStream_t st) {
    static_assert(sizeof(K) == 4 || sizeof(K) == 8, "u32 or u64 keys");
    if (end_bit > 8 * (int)sizeof(K)) end_bit = 8 * (int)sizeof(K);
    if (n <= 1 || end_bit <= begin_bit) return 0;
    const int npasses = (end_bit - begin_bit + RS_BITS - 1) / RS_BITS;
    auto m = A.mark();
    unsigned long long* hist = A.alloc<unsigned long long>((size_t)npasses * RS_BINS);
    CDBG_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * npasses * RS_BINS, st));
    {
        uint64_t blocks = ceil_div(n, (uint64_t)RS_THREADS * 16);
        if (blocks > 148 * 8) blocks = 148 * 8;
        {
            CDBG_PROF("k_rs_histograms", st);
            k_rs_histograms<<<(unsigned)blocks, RS_THREADS, 0, st>>>(keys, n, begin_bit, npasses, hist);
        }
        CDBG_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> h((size_t)npasses * RS_BINS);
    read_small(h.data(), hist, h.size() * 8, st);

    const uint64_t ntiles = ceil_div(n, RS_TILE);
    K* k2 = A.alloc<K>(n);
    V* v2 = A.alloc<V>(n);
    uint32_t* counts = A.alloc<uint32_t>(ntiles * RS_BINS);
    uint64_t* offs = A.alloc<uint64_t>(ntiles * RS_BINS);
    K *kin = keys, *kout = k2;
    V *vin = vals, *vout = v2;
    int ran = 0;
    for (int p = 0; p < npasses; ++p) {
        bool trivial = false;
        for (int d = 0; d < RS_BINS; ++d)
            if (h[(size_t)p * RS_BINS + d] == n) trivial = true;
        if (trivial) continue;
        const int shift = begin_bit + p * RS_BITS;
        {
            CDBG_PROF("k_rs_upsweep", st);
            k_rs_upsweep<<<(unsigned)ntiles, RS_THREADS, 0, st>>>(kin, n, shift, (uint32_t)ntiles, counts);
        }
        CDBG_CHECK_LAUNCH();
        exclusive_scan<uint32_t, uint64_t>(counts, offs, ntiles * RS_BINS, A, st);
        {
            // one read and one write of every (key, value) pair
            CDBG_PROF_BYTES("k_rs_downsweep", st, 2.0 * n * (sizeof(K) + sizeof(V)));
            k_rs_downsweep<K, V><<<(unsigned)ntiles, RS_THREADS, 0, st>>>(kin, vin, kout, vout, n, shift,
                                                                       (uint32_t)ntiles, offs);
        }
        CDBG_CHECK_LAUNCH();
        std::swap(kin, kout);
        std::swap(vin, vout);
        ++ran;
    }
    if (kin != keys) {
        CDBG_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(K), cudaMemcpyDeviceToDevice, st));
        CDBG_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(V), cudaMemcpyDeviceToDevice, st));
    }
    A.release(m);
    return ran;
}

}  // namespace
}  // namespace prim
}  // namespace cdbg
