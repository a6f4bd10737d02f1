// Device-wide primitives written for this project: exclusive scan and a
// stable LSD radix sort of (key, value) pairs, u32 or u64 keys.
//
// Radix sort: one fused histogram pass computes the digit histograms of every
// requested pass in a single read of the keys; passes whose digit is constant
// over all keys are skipped.  Each executed pass is ONE kernel (k_rs_onesweep):
// tiles rank their keys stably with warp match-any, find their global digit
// offsets by a decoupled look-back per digit, stage the tile in shared memory
// in digit order and write each digit's run contiguously.
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
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_WARPS = RS_THREADS / 32;

// One pass of the LSD sort in a single kernel (decoupled look-back per
// digit).  Tiles take their indices in launch order from *tile_counter, so
// every predecessor of a tile is running or done.  A tile ranks its keys
// stably (warp w owns positions [w*ITEMS*32, (w+1)*ITEMS*32), processed in
// rounds of 32 with warp match-any), publishes its per-digit counts in
// status[tile][d], walks back over its predecessors' entries of the same digit
// until an inclusive prefix (one thread per digit), publishes its own
// inclusive prefix, stages the tile in shared memory in digit order and writes
// each digit's run contiguously at digit_start[d] + prefix.  Status words are
// [flag:2 | epoch:4 | count:58]; the epoch is the pass number, so one zeroing
// per sort serves every pass.  Waits are bounded: a tile that gives up sets
// *err and publishes what it has, so no successor waits on it, and its
// successors' positions can only come out smaller than the true ones, which
// keeps every write inside the output.
constexpr unsigned long long RS_AGG = 1ull << 62, RS_INC = 2ull << 62, RS_VALMASK = (1ull << 58) - 1;

template <int BITS, int ITEMS, typename K, typename V>
struct rs_smem {
    static constexpr int BINS = 1 << BITS;
    static constexpr int TILE = RS_THREADS * ITEMS;
    K sk[TILE];
    V sv[TILE];
    uint32_t wcnt[RS_WARPS][BINS];  // per-warp digit counts, then prefixes
    uint32_t dstart[BINS];          // tile-local start of each digit
    uint64_t gbase[BINS];           // global start of each digit for this tile
    uint32_t sw[RS_WARPS + 1];
    uint32_t tile;
};

template <int BITS, int ITEMS, typename K, typename V>
__global__ void __launch_bounds__(RS_THREADS, 3) k_rs_onesweep(K const* __restrict__ keys_in,
                                                            V const* __restrict__ vals_in,
                                                            K* __restrict__ keys_out, V* __restrict__ vals_out,
                                                            uint64_t n, int shift, uint32_t* tile_counter,
                                                            unsigned long long* status,
                                                            unsigned long long const* __restrict__ digit_start,
                                                            uint32_t epoch, uint32_t* err) {
    using S = rs_smem<BITS, ITEMS, K, V>;
    constexpr int BINS = S::BINS, TILE = S::TILE, DPT = (BINS + RS_THREADS - 1) / RS_THREADS;
    extern __shared__ __align__(16) unsigned char rs_raw[];
    S& sm = *reinterpret_cast<S*>(rs_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_WARPS * BINS; i += RS_THREADS) (&sm.wcnt[0][0])[i] = 0;
    if (threadIdx.x == 0) sm.tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = sm.tile;
    const uint64_t base = tile * TILE;
    const uint32_t tile_n = (uint32_t)((n - base) < (uint64_t)TILE ? (n - base) : TILE);
    K k[ITEMS];
    V v[ITEMS];
    uint32_t rk[ITEMS];
#pragma unroll
    for (int r = 0; r < ITEMS; ++r) {
        const uint32_t pos = (uint32_t)warp * (ITEMS * 32) + (uint32_t)r * 32 + lane;
        const bool ok = pos < tile_n;
        k[r] = ok ? keys_in[base + pos] : ~K(0);
        v[r] = ok ? vals_in[base + pos] : V(0);
    }
#pragma unroll
    for (int r = 0; r < ITEMS; ++r) {
        const uint32_t pos = (uint32_t)warp * (ITEMS * 32) + (uint32_t)r * 32 + lane;
        const bool ok = pos < tile_n;
        const uint32_t d = ok ? (uint32_t)((k[r] >> shift) & (BINS - 1)) : BINS;  // sentinel
        const uint32_t active = __ballot_sync(0xffffffffu, ok);
        const uint32_t peers = __match_any_sync(0xffffffffu, d) & active;
        uint32_t old = 0;
        const int leader = peers ? __ffs(peers) - 1 : 0;
        if (ok && lane == leader) {
            old = sm.wcnt[warp][d];
            sm.wcnt[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rk[r] = ok ? old + __popc(peers & lanemask_lt()) : 0;
    }
    __syncthreads();
    // per digit: exclusive prefix over warps and the tile's count
    uint32_t cnt[DPT];
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
        const int d = threadIdx.x + j * RS_THREADS;
        uint32_t run = 0;
        if (d < BINS) {
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) {
                const uint32_t c = sm.wcnt[w][d];
                sm.wcnt[w][d] = run;
                run += c;
            }
            const unsigned long long ep = (unsigned long long)epoch << 58;
            *(volatile unsigned long long*)&status[tile * BINS + d] = (tile == 0 ? RS_INC : RS_AGG) | ep | run;
        }
        cnt[j] = run;
    }
    // look-back, one thread per digit
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
        const int d = threadIdx.x + j * RS_THREADS;
        if (d >= BINS) continue;
        uint64_t excl = 0;
        if (tile > 0) {
            bool ok = true;
            for (uint64_t t = tile - 1;; --t) {
                unsigned long long w = 0;
                uint32_t spin = 0;
                for (; spin < (1u << 24); ++spin) {
                    w = *(volatile unsigned long long*)&status[t * BINS + d];
                    if ((w >> 62) != 0 && ((w >> 58) & 15u) == epoch) break;
                }
                if (spin == (1u << 24)) {
                    ok = false;
                    break;
                }
                excl += w & RS_VALMASK;
                if ((w >> 62) == 2 || t == 0) break;
            }
            if (!ok) set_error(err, ERR_CHAIN_LIMIT);
            const unsigned long long ep = (unsigned long long)epoch << 58;
            *(volatile unsigned long long*)&status[tile * BINS + d] = RS_INC | ep | ((excl + cnt[j]) & RS_VALMASK);
        }
        sm.gbase[d] = digit_start[d] + excl;
    }
    // tile-local digit starts (exclusive scan of the counts over digits)
    {
        // thread t owns digits t, t + RS_THREADS, ...: one block scan per
        // column keeps the starts in digit order
        uint32_t carry = 0;
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            uint32_t tot;
            const uint32_t ex = block_exclusive_scan<uint32_t, RS_THREADS>(cnt[j], sm.sw, tot);
            const int d = threadIdx.x + j * RS_THREADS;
            if (d < BINS) sm.dstart[d] = carry + ex;
            carry += tot;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < ITEMS; ++r) {
        const uint32_t pos = (uint32_t)warp * (ITEMS * 32) + (uint32_t)r * 32 + lane;
        if (pos < tile_n) {
            const uint32_t d = (uint32_t)((k[r] >> shift) & (BINS - 1));
            const uint32_t lp = sm.dstart[d] + sm.wcnt[warp][d] + rk[r];
            sm.sk[lp] = k[r];
            sm.sv[lp] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < tile_n; p += RS_THREADS) {
        const K key = sm.sk[p];
        const uint32_t d = (uint32_t)((key >> shift) & (BINS - 1));
        const uint64_t dst = sm.gbase[d] + (p - sm.dstart[d]);
        if (dst < n) {
            keys_out[dst] = key;
            vals_out[dst] = sm.sv[p];
        }
    }
}

// Exclusive scan of each pass's digit histogram: starts[p][d].
template <int BITS>
__global__ void k_rs_digit_starts(unsigned long long const* __restrict__ hist, int npasses,
                                  unsigned long long* __restrict__ starts) {
    constexpr int BINS = 1 << BITS;
    const int p = blockIdx.x;
    if (p >= npasses || threadIdx.x != 0) return;
    unsigned long long run = 0;
    for (int d = 0; d < BINS; ++d) {
        starts[(size_t)p * BINS + d] = run;
        run += hist[(size_t)p * BINS + d];
    }
}

// Histograms of all passes with BITS-bit digits, in one read.  hist is
// npasses x 2^BITS u64, zeroed by the caller.
template <int BITS, typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_histograms_w(K const* __restrict__ keys, uint64_t n,
                                                                int begin_bit, int npasses,
                                                                unsigned long long* hist) {
    constexpr int BINS = 1 << BITS;
    extern __shared__ uint32_t hw[];  // npasses x BINS
    for (int i = threadIdx.x; i < npasses * BINS; i += RS_THREADS) hw[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * RS_THREADS;
    for (uint64_t i = (uint64_t)blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += stride) {
        const K k = keys[i];
        for (int p = 0; p < npasses; ++p) atomicAdd(&hw[p * BINS + ((k >> (begin_bit + p * BITS)) & (BINS - 1))], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * BINS; i += RS_THREADS) {
        const uint32_t v = hw[i];
        if (v) atomicAdd(&hist[i], (unsigned long long)v);
    }
}

template <int BITS, typename V, typename K>
int radix_sort_pairs_w(K* keys, V* vals, uint64_t n, int begin_bit, int end_bit, dev_arena& A,
                       cudaStream_t st, uint32_t* err) {
    constexpr int BINS = 1 << BITS;
    constexpr int ITEMS = 16;
    using S = rs_smem<BITS, ITEMS, K, V>;
    constexpr int TILE = S::TILE;
    const int npasses = (end_bit - begin_bit + BITS - 1) / BITS;
    if (npasses > 15) throw std::runtime_error("radix sort: too many passes");
    auto m = A.mark();
    unsigned long long* hist = A.alloc<unsigned long long>((size_t)npasses * BINS);
    unsigned long long* starts = A.alloc<unsigned long long>((size_t)npasses * BINS);
    CDBG_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * npasses * BINS, st));
    {
        uint64_t blocks = ceil_div(n, (uint64_t)RS_THREADS * 16);
        if (blocks > 148 * 8) blocks = 148 * 8;
        const size_t hs = sizeof(uint32_t) * npasses * BINS;
        if (hs > 48 * 1024)
            CDBG_CUDA(cudaFuncSetAttribute(k_rs_histograms_w<BITS, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)hs));
        {
            CDBG_PROF("k_rs_histograms", st);
            k_rs_histograms_w<BITS, K><<<(unsigned)blocks, RS_THREADS, hs, st>>>(keys, n, begin_bit, npasses, hist);
        }
        CDBG_CHECK_LAUNCH();
        k_rs_digit_starts<BITS><<<npasses, 32, 0, st>>>(hist, npasses, starts);
        CDBG_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> h((size_t)npasses * BINS);
    read_small(h.data(), hist, h.size() * 8, st);

    const uint64_t ntiles = ceil_div(n, (uint64_t)TILE);
    K* k2 = A.alloc<K>(n);
    V* v2 = A.alloc<V>(n);
    unsigned long long* status = A.alloc<unsigned long long>(ntiles * BINS);
    uint32_t* counters = A.alloc<uint32_t>(npasses);
    CDBG_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned long long) * ntiles * BINS, st));
    CDBG_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * npasses, st));
    CDBG_CUDA(cudaFuncSetAttribute(k_rs_onesweep<BITS, ITEMS, K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sizeof(S)));
    K *kin = keys, *kout = k2;
    V *vin = vals, *vout = v2;
    int ran = 0;
    for (int p = 0; p < npasses; ++p) {
        bool trivial = false;
        for (int d = 0; d < BINS; ++d)
            if (h[(size_t)p * BINS + d] == n) trivial = true;
        if (trivial) continue;
        const int shift = begin_bit + p * BITS;
        {
            // one read and one write of every (key, value) pair
            CDBG_PROF_BYTES("k_rs_onesweep", st, 2.0 * n * (sizeof(K) + sizeof(V)));
            k_rs_onesweep<BITS, ITEMS, K, V><<<(unsigned)ntiles, RS_THREADS, sizeof(S), st>>>(
                kin, vin, kout, vout, n, shift, counters + p, status, starts + (size_t)p * BINS, (uint32_t)(p + 1),
                err);
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

// Stable sort of (keys, vals) by key bits [begin_bit, end_bit) with 8-bit or
// 11-bit digits (g_radix_bits: the engine's tuning; 11 bits take 3 passes
// where 8 bits take 4, with 8x the counters and look-back state per tile).
// Results end in (keys, vals); the arena provides the ping-pong buffers.
// Needs a host synchronize (to read the digit histograms); returns the number
// of passes run.  A look-back that gives up sets *err.
template <typename V, typename K = uint64_t>
int radix_sort_pairs(K* keys, V* vals, uint64_t n, int begin_bit, int end_bit, dev_arena& A, cudaStream_t st,
                     uint32_t* err) {
    static_assert(sizeof(K) == 4 || sizeof(K) == 8, "u32 or u64 keys");
    if (end_bit > 8 * (int)sizeof(K)) end_bit = 8 * (int)sizeof(K);
    if (n <= 1 || end_bit <= begin_bit) return 0;
    if (g_radix_bits == 11) return radix_sort_pairs_w<11, V, K>(keys, vals, n, begin_bit, end_bit, A, st, err);
    return radix_sort_pairs_w<RS_BITS, V, K>(keys, vals, n, begin_bit, end_bit, A, st, err);
}

// ----------------------------------------- exact 64-bit order, 32-bit passes
// Keys whose top 32 bits tie but whose full keys differ, after a stable sort
// on the top 32 bits: positions i with hi(i) == hi(i - 1), key(i) != key(i - 1)
// appended to `list` (count in *cnt, at most `cap` stored).
__global__ void k_hi_mismatch(uint64_t const* __restrict__ keys, uint64_t n, uint32_t* __restrict__ list,
                              unsigned long long* cnt, uint64_t cap) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool m = false;
    if (i > 0 && i < n) {
        const uint64_t a = keys[i - 1], b = keys[i];
        m = (a >> 32) == (b >> 32) && a != b;
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, m);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(bal) - 1) base = atomicAdd(cnt, (unsigned long long)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
    if (m) {
        const uint64_t o = base + __popc(bal & lanemask_lt());
        if (o < cap) list[o] = (uint32_t)i;
    }
}

__device__ __forceinline__ uint64_t hi_lower_bound(uint64_t const* keys, uint64_t lo, uint64_t hi, uint32_t h) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if ((uint32_t)(keys[mid] >> 32) < h)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// For each (sorted) mismatch position: the run of its top 32 bits [s, e),
// and whether it is the run's first mismatch (the run's representative).
__global__ void k_hi_runs(uint64_t const* __restrict__ keys, uint64_t n, uint32_t const* __restrict__ list,
                          uint64_t nm, uint64_t* __restrict__ rs, uint64_t* __restrict__ len) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nm) return;
    const uint64_t i = list[j];
    const uint32_t h = (uint32_t)(keys[i] >> 32);
    const uint64_t s = hi_lower_bound(keys, 0, i, h);
    const uint64_t e = h == 0xffffffffu ? n : hi_lower_bound(keys, i, n, h + 1);
    const bool rep = j == 0 || list[j - 1] < s;
    rs[j] = s;
    len[j] = rep ? e - s : 0;
}

__device__ __forceinline__ uint64_t upper_bound_off(uint64_t const* a, uint64_t n, uint64_t x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Compact element j of the mixed runs: run r (by its compact offset) and its
// position in the full array.
__device__ __forceinline__ uint64_t hi_pos(uint64_t const* off, uint64_t const* rs, uint64_t nm, uint64_t j,
                                           uint64_t& r) {
    // the last entry starting at or before j; entries that are not their
    // run's representative have length 0 and follow it, so they start after j
    r = upper_bound_off(off, nm + 1, j) - 1;
    return rs[r] + (j - off[r]);
}

__global__ void k_hi_gather_keys(uint64_t const* __restrict__ keys, uint64_t const* __restrict__ off,
                                 uint64_t const* __restrict__ rs, uint64_t nm, uint64_t M,
                                 uint64_t* __restrict__ ckey, uint32_t* __restrict__ cpos) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    uint64_t r;
    const uint64_t q = hi_pos(off, rs, nm, j, r);
    ckey[j] = ((uint64_t)r << 32) | (uint32_t)keys[q];
    cpos[j] = (uint32_t)q;
}

template <typename V>
__global__ void k_hi_permute(uint64_t const* __restrict__ keys, V const* __restrict__ vals,
                             uint32_t const* __restrict__ cpos, uint64_t M, uint64_t* __restrict__ tk,
                             V* __restrict__ tv) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    tk[j] = keys[cpos[j]];
    tv[j] = vals[cpos[j]];
}

template <typename V>
__global__ void k_hi_scatter(uint64_t* __restrict__ keys, V* __restrict__ vals, uint64_t const* __restrict__ off,
                             uint64_t const* __restrict__ rs, uint64_t nm, uint64_t M,
                             uint64_t const* __restrict__ tk, V const* __restrict__ tv) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    uint64_t r;
    const uint64_t q = hi_pos(off, rs, nm, j, r);
    keys[q] = tk[j];
    vals[q] = tv[j];
}

// Stable sort of (u64 keys, vals) by all 64 key bits -- the same order as an
// 8-pass LSD sort -- in 4 passes over the top 32 bits: keys that tie on those
// bits but differ below them (rare when the top bits are a hash) are found
// afterwards, and only their runs are sorted again on (run, low 32 bits).
// n < 2^32.
template <typename V>
void sort_pairs_u64_exact(uint64_t* keys, V* vals, uint64_t n, dev_arena& A, cudaStream_t st, uint32_t* err) {
    if (n <= 1) return;
    if (n >= (1ull << 32)) throw std::runtime_error("sort_pairs_u64_exact: n >= 2^32");
    radix_sort_pairs<V, uint64_t>(keys, vals, n, 32, 64, A, st, err);
    auto m = A.mark();
    const uint64_t cap = n / 8 + 1024;
    uint32_t* list = A.alloc<uint32_t>(cap);
    unsigned long long* cnt = A.alloc<unsigned long long>(1);
    CDBG_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
    {
        CDBG_PROF("k_hi_mismatch", st);
        k_hi_mismatch<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(keys, n, list, cnt, cap);
    }
    CDBG_CHECK_LAUNCH();
    unsigned long long nm = 0;
    read_small(&nm, cnt, 8, st);
    if (nm > cap) {
        // far from a hash: the full stable sort of the (already top-sorted)
        // pairs gives the same order as sorting the input
        A.release(m);
        radix_sort_pairs<V, uint64_t>(keys, vals, n, 0, 64, A, st, err);
        return;
    }
    if (nm == 0) {
        A.release(m);
        return;
    }
    uint32_t* dummy = A.alloc<uint32_t>(nm);
    radix_sort_pairs<uint32_t, uint32_t>(list, dummy, nm, 0, 32, A, st, err);
    uint64_t* rs = A.alloc<uint64_t>(nm);
    uint64_t* len = A.alloc<uint64_t>(nm);
    uint64_t* off = A.alloc<uint64_t>(nm + 1);
    k_hi_runs<<<(unsigned)ceil_div(nm, 256), 256, 0, st>>>(keys, n, list, nm, rs, len);
    CDBG_CHECK_LAUNCH();
    exclusive_scan<uint64_t, uint64_t>(len, off, nm, A, st, off + nm);
    uint64_t M = 0;
    read_small(&M, off + nm, 8, st);
    uint64_t* ckey = A.alloc<uint64_t>(M);
    uint32_t* cpos = A.alloc<uint32_t>(M);
    k_hi_gather_keys<<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(keys, off, rs, nm, M, ckey, cpos);
    CDBG_CHECK_LAUNCH();
    int rb = 1;
    while ((1ull << rb) < nm) ++rb;
    radix_sort_pairs<uint32_t, uint64_t>(ckey, cpos, M, 0, 32 + rb, A, st, err);
    uint64_t* tk = A.alloc<uint64_t>(M);
    V* tv = A.alloc<V>(M);
    k_hi_permute<V><<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(keys, vals, cpos, M, tk, tv);
    CDBG_CHECK_LAUNCH();
    k_hi_scatter<V><<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(keys, vals, off, rs, nm, M, tk, tv);
    CDBG_CHECK_LAUNCH();
    A.release(m);
}

}  // namespace
}  // namespace prim
}  // namespace cdbg
