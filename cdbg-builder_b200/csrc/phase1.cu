// Phase 1 (bucket-write) kernels for sm_100a.
//
// Restates on the device what the reference does per input file in
// phase1_bucket_write/bucket_ingester.hpp:36-177 and the compaction of
// bucket_io.hpp:127-277:
//   1. ACGT runs >= k of every sequence (bucket_ingester.hpp:152-171),
//      packed into a 2-bit stream (one 64-bit word = 32 bases).
//   2. Per run tile (2048 (k-1)-mers, staged into shared memory with a TMA
//      bulk copy): canonical ntHash of each m-mer (minimizer.hpp:40-62),
//      sliding minimum over W = k - m m-mers = the (k-1)-mer minimizer
//      (minimizer.hpp:94-157), and the super-k-mer cut points where the
//      minimizer changes (bucket_ingester.hpp:106-126).
//   3. Super-k-mers with flags, bucket (h >> 1) % B and a 64-bit key hash.
//   4. Full per-bucket dedup: stable radix sort by (bucket, key hash), equal
//      neighbours merged (flags AND, colors sorted-unique) -- the merge rule of
//      bucket_io.hpp:137-166, applied to the whole bucket instead of a spill
//      window (phase-2 results do not depend on the window).
//   5. Record serialization in the bucket-file record layout
//      (super_kmer.hpp:105-117) and the inverse parse (super_kmer.hpp:121-143).

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>
#include <mutex>
#include <string>
#include <vector>

#include "device_kmer.cuh"
#include "phase1.cuh"
#include "primitives.cuh"

namespace cdbg {

namespace {

constexpr int EV_THREADS = 256;
constexpr int EV_PER_THREAD = 32;
constexpr int EV_TILE = EV_THREADS * EV_PER_THREAD;

__device__ __forceinline__ uint32_t nuc_code(uint8_t c) {
    // A/a=0 C/c=1 G/g=2 T/t=3 else 0xff (kmer.hpp:35-52)
    switch (c | 0x20) {
        case 'a': return 0;
        case 'c': return 1;
        case 'g': return 2;
        case 't': return 3;
        default: return 0xffu;
    }
}

__device__ __forceinline__ uint32_t upper_bound_u64(uint64_t const* a, uint32_t n, uint64_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t byte_valid(uint32_t c) {
    const uint32_t l = c | 0x20u;
    return (l == 'a' || l == 'c' || l == 'g' || l == 't') ? 1u : 0u;
}

// Boundary bitmap of the input: bit p set for every sequence start p and for
// p = nbytes (seq_off[num_seqs]), one thread per offset.
__global__ void k_seq_starts(uint64_t const* __restrict__ seq_off, uint32_t num_seqs, uint32_t* __restrict__ bits) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s > num_seqs) return;
    const uint64_t p = seq_off[s];
    atomicOr(&bits[p >> 5], 1u << (uint32_t)(p & 31));
}

// Run boundary events over positions [0, nbytes]: (pos << 1) | 1 for a run
// start, (pos << 1) for a run end.  Sequence starts (and nbytes) split runs.
// Each thread owns 32 positions as bit masks: V = valid bases, S = sequence
// starts, P = validity of the byte before each position; then
//   ends   = P & (~V | S)
//   starts = V & (S | ~P)
// (a full 32-byte chunk is read with two 16-byte loads when aligned).
// Run boundaries at positions [p0, p0 + 32) as bit masks: E (a run ends at
// p) and St (a run starts at p).
__device__ __forceinline__ void ev_masks(uint8_t const* __restrict__ ascii, uint64_t nbytes,
                                         uint32_t const* __restrict__ starts, uint64_t p0, uint32_t& E,
                                         uint32_t& St) {
    E = St = 0;
    if (p0 > nbytes) return;
    uint32_t V = 0;
    if (p0 + 32 <= nbytes && ((reinterpret_cast<uintptr_t>(ascii) & 15) == 0)) {
        const uint4 a = reinterpret_cast<uint4 const*>(ascii + p0)[0];
        const uint4 b = reinterpret_cast<uint4 const*>(ascii + p0)[1];
        const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 32; ++i) V |= byte_valid((w[i >> 2] >> (8 * (i & 3))) & 0xffu) << i;
    } else {
        const uint32_t n = (uint32_t)((nbytes - p0) < 32 ? (nbytes - p0) : 32);
        for (uint32_t i = 0; i < n; ++i) V |= byte_valid(ascii[p0 + i]) << i;
    }
    // sequence starts in [p0, p0 + 32), and nbytes itself (bit i of word
    // p0 / 32 of the boundary bitmap; p0 is a multiple of 32)
    const uint32_t S = starts[p0 >> 5];
    // validity of the byte before p0, whatever sequence it belongs to: a
    // run of the previous sequence that ends exactly at p0 is closed here
    const uint32_t pin = (p0 > 0) ? byte_valid(ascii[p0 - 1]) : 0u;
    const uint32_t P = (V << 1) | pin;
    E = P & (~V | S);
    St = V & (S | ~P);
    if (nbytes - p0 < 31) {  // positions past nbytes are not positions
        const uint32_t keep = (2u << (uint32_t)(nbytes - p0)) - 1u;
        E &= keep;
        St &= keep;
    }
}

__device__ __forceinline__ void ev_write(uint32_t E, uint32_t St, uint64_t p0, uint64_t o, uint64_t cap,
                                         uint64_t* __restrict__ events) {
    uint32_t m = E | St;
    while (m) {
        const uint32_t i = __ffs(m) - 1;
        m &= m - 1;
        const uint64_t p = p0 + i;
        if ((E >> i) & 1u) {  // run end
            if (o < cap) events[o] = p << 1;
            ++o;
        }
        if ((St >> i) & 1u) {  // run start
            if (o < cap) events[o] = (p << 1) | 1u;
            ++o;
        }
    }
}

// Run boundary events over positions [0, nbytes]: (pos << 1) | 1 for a run
// start, (pos << 1) for a run end.  Sequence starts (and nbytes) split runs.
// Each thread owns 32 positions as bit masks: V = valid bases, S = sequence
// starts, P = validity of the byte before each position; then
//   ends   = P & (~V | S)
//   starts = V & (S | ~P)
// (a full 32-byte chunk is read with two 16-byte loads when aligned).
// Two passes: the counts per tile, then (after their scan) the events.
template <bool WRITE>
__global__ void __launch_bounds__(EV_THREADS)
    k_run_events(uint8_t const* __restrict__ ascii, uint64_t nbytes, uint32_t const* __restrict__ starts,
                 uint32_t* __restrict__ tile_count, uint64_t const* __restrict__ tile_off,
                 uint64_t* __restrict__ events) {
    static_assert(EV_PER_THREAD == 32, "one 32-bit mask per thread");
    __shared__ uint32_t sw[EV_THREADS / 32 + 1];
    const uint64_t p0 = (uint64_t)blockIdx.x * EV_TILE + (uint64_t)threadIdx.x * EV_PER_THREAD;
    uint32_t E, St;
    ev_masks(ascii, nbytes, starts, p0, E, St);
    const uint32_t cnt = __popc(E) + __popc(St);
    uint32_t tot;
    const uint32_t ex = prim::block_exclusive_scan<uint32_t, EV_THREADS>(cnt, sw, tot);
    if (!WRITE) {
        if (threadIdx.x == 0) tile_count[blockIdx.x] = tot;
        return;
    }
    ev_write(E, St, p0, tile_off[blockIdx.x] + ex, ~0ull, events);
}

// The same in one pass: tiles take indices in launch order and find their
// output offset by decoupled look-back; events past `cap` are counted, not
// written, and the last tile stores the total in *total (the caller runs the
// two passes when it exceeds cap).
__global__ void __launch_bounds__(EV_THREADS)
    k_run_events_1p(uint8_t const* __restrict__ ascii, uint64_t nbytes, uint32_t const* __restrict__ starts,
                    uint64_t ntiles, uint32_t* tile_counter, unsigned long long* status,
                    uint64_t* __restrict__ events, uint64_t cap, unsigned long long* total, uint32_t* err) {
    __shared__ uint32_t sw[EV_THREADS / 32 + 1];
    __shared__ uint64_t s_tile, s_excl;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t p0 = tile * EV_TILE + (uint64_t)threadIdx.x * EV_PER_THREAD;
    uint32_t E, St;
    ev_masks(ascii, nbytes, starts, p0, E, St);
    const uint32_t cnt = __popc(E) + __popc(St);
    uint32_t tot;
    const uint32_t ex = prim::block_exclusive_scan<uint32_t, EV_THREADS>(cnt, sw, tot);
    if (threadIdx.x < 32) {
        uint64_t excl = 0;
        const bool ok = prim::lookback_exclusive(status, tile, tot, excl);
        if (threadIdx.x == 0) {
            if (!ok) set_error(err, ERR_CHAIN_LIMIT);
            s_excl = excl;
            if (tile == ntiles - 1) *total = excl + tot;
        }
    }
    __syncthreads();
    ev_write(E, St, p0, s_excl + ex, cap, events);
}

// Pair events into runs; keep[i] = len >= k.
__global__ void k_runs_from_events(uint64_t const* __restrict__ ev, uint64_t nruns,
                                   uint64_t const* __restrict__ seq_off, uint32_t num_seqs,
                                   uint32_t const* __restrict__ seq_color, uint32_t k,
                                   uint64_t* __restrict__ src, uint32_t* __restrict__ len,
                                   uint32_t* __restrict__ color, uint32_t* __restrict__ keep,
                                   uint32_t* err) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nruns) return;
    const uint64_t a = ev[2 * i] >> 1, b = ev[2 * i + 1] >> 1;
    const uint64_t l = b - a;
    if (l >= 0xffffffffull) set_error(err, ERR_FIELD_OVERFLOW);
    src[i] = a;
    len[i] = (uint32_t)l;
    uint32_t s = upper_bound_u64(seq_off, num_seqs + 1, a) - 1;
    color[i] = seq_color[s];
    keep[i] = l >= k ? 1u : 0u;
}

__global__ void k_runs_compact(uint64_t nruns, uint32_t const* __restrict__ keep,
                               uint64_t const* __restrict__ kpos, uint64_t const* __restrict__ src,
                               uint32_t const* __restrict__ len, uint32_t const* __restrict__ color,
                               uint64_t* __restrict__ osrc, uint32_t* __restrict__ olen,
                               uint32_t* __restrict__ ocolor, uint64_t* __restrict__ padded) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nruns || !keep[i]) return;
    const uint64_t o = kpos[i];
    osrc[o] = src[i];
    olen[o] = len[i];
    ocolor[o] = color[i];
    padded[o] = ((uint64_t)len[i] + 31) & ~uint64_t(31);
}

// One 64-bit stream word per thread.
__global__ void k_pack(uint8_t const* __restrict__ ascii, uint32_t nruns,
                       uint64_t const* __restrict__ soff, uint64_t const* __restrict__ src,
                       uint32_t const* __restrict__ len, uint64_t nwords_data,
                       uint64_t* __restrict__ words) {
    uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwords_data) return;
    const uint64_t pos = w * 32;
    const uint32_t r = upper_bound_u64(soff, nruns, pos) - 1;
    const uint64_t j = pos - soff[r];
    const uint32_t L = len[r];
    uint64_t out = 0;
    if (j < L) {
        const uint32_t n = (L - j) < 32 ? (uint32_t)(L - j) : 32u;
        uint8_t const* p = ascii + src[r] + j;
        for (uint32_t i = 0; i < n; ++i) out |= (uint64_t)(nuc_code(p[i]) & 3u) << (2 * i);
    }
    words[w] = out;
}

// ------------------------------------------------------------ minimizer tile
constexpr int MZ_THREADS = 256;
constexpr int MZ_TT = 2048;  // default (k-1)-mers per tile

__device__ __forceinline__ uint32_t smem_u32(void const* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// TMA bulk copy global -> shared (cp.async.bulk), completion on an mbarrier.
// The wait is bounded; on a timeout the whole block gets false and the error
// word is set (the block then exits without touching the staged tile).
__device__ __forceinline__ bool tma_load_1d(void* smem_dst, void const* gsrc, uint32_t bytes,
                                            uint64_t* bar, uint32_t* err) {
    const uint32_t b = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(smem_dst)),
            "l"(gsrc), "r"(bytes), "r"(b)
            : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(b)
            : "memory");
        if (done) break;
    }
    const int ok = __syncthreads_and((int)done);
    if (!ok && threadIdx.x == 0) set_error(err, ERR_CHAIN_LIMIT);
    return ok != 0;
}

// Shared memory of one minimizer tile of TT (k-1)-mers: the staged 2-bit
// words, the m-mer hashes (padded one slot per 32 so that threads hashing
// consecutive chunks store to different banks) and the per-position minima.
template <int TT>
struct mz_layout {
    static constexpr int WMAX = (TT + 256) / 32 + 4;       // 2-bit words staged
    static constexpr int HMAX = TT + 1 + 64;               // m-mer hashes (W <= 62)
    static constexpr int HPAD = HMAX + HMAX / 32 + 1;
    static constexpr size_t bytes = sizeof(uint64_t) * (WMAX + HPAD + TT + 1);
};
__device__ __forceinline__ uint32_t mz_pad(uint32_t q) { return q + (q >> 5); }

// 32 bases starting at stream offset x of the staged words (base x in the
// low two bits).
__device__ __forceinline__ uint64_t mz_window(uint64_t const* sw, uint32_t x) {
    const uint64_t lo = sw[x >> 5], hi = sw[(x >> 5) + 1];
    const uint32_t s = 2 * (x & 31);
    return s ? (lo >> s) | (hi << (64 - s)) : lo;
}

// Rolling-hash tables of one tile, filled by threads 0..63: stab[j][b] =
// [0] seed(b), [1] rol(seed(b), m), [2] ror(seed(b^3), 1), [3] rol(seed(b^3),
// m-1); tf/tr[(out << 2) | in] = one rolling step of base `out` leaving and
// base `in` entering, forward and reverse-complement strand; and, for the
// first m-mer of a chunk two bases at a time, p2f[x] = rol(seed(a), 1) ^
// seed(b) and p2r[x] = rol(seed(b ^ 3), 1) ^ seed(a ^ 3) for the base pair x =
// a | b << 2 (a first in the sequence).
__device__ __forceinline__ void mz_tables(uint64_t (*stab)[4], uint64_t* tf, uint64_t* tr, uint64_t* p2f,
                                          uint64_t* p2r, uint32_t m) {
    if (threadIdx.x >= 32 && threadIdx.x < 64) {
        const uint32_t x = threadIdx.x & 15, a = x & 3, b = x >> 2;
        if (threadIdx.x < 48)
            p2f[x] = rol64(nt_seed(a), 1) ^ nt_seed(b);
        else
            p2r[x] = rol64(nt_seed(b ^ 3u), 1) ^ nt_seed(a ^ 3u);
    }
    if (threadIdx.x < 16) {
        const uint32_t b = threadIdx.x & 3, j = threadIdx.x >> 2;
        const uint64_t sb = nt_seed(b), sc = nt_seed(b ^ 3u);
        stab[j][b] = j == 0 ? sb : j == 1 ? rol64(sb, m) : j == 2 ? ror64(sc, 1) : rol64(sc, m - 1);
    } else if (threadIdx.x < 32) {
        const uint32_t o = (threadIdx.x - 16) >> 2, i = threadIdx.x & 3;
        tf[(o << 2) | i] = rol64(nt_seed(o), m) ^ nt_seed(i);
        tr[(o << 2) | i] = ror64(nt_seed(o ^ 3u), 1) ^ rol64(nt_seed(i ^ 3u), m - 1);
    }
}

// Canonical m-mer hashes h[0..nh) of a staged tile (h[q] = the m-mer at
// stream offset rel0 + q of sw) into sh[mz_pad(q)]: thread c hashes the HC
// m-mers from c * HC on, the first in Horner form (fwd = xor_i rol(seed(b_i),
// m-1-i), rc = xor_i rol(seed(b_i ^ 3), i)), the others rolled with one
// (out, in) table entry per strand.  Its bases sit in two 32-base register
// windows, so every extraction in the unrolled loop is a constant shift.
template <int HC>
__device__ __forceinline__ void mz_hash(uint64_t const* sw, uint64_t* sh, uint64_t const (*stab)[4],
                                        uint64_t const* tf, uint64_t const* tr, uint64_t const* p2f,
                                        uint64_t const* p2r, uint32_t rel0, uint32_t nh, uint32_t m) {
    const uint32_t q0 = threadIdx.x * HC;
    if (q0 >= nh) return;
    const uint32_t cnt = min((uint32_t)HC, nh - q0);
    const uint32_t x0 = rel0 + q0;
    const uint64_t wout = mz_window(sw, x0);         // bases q0 .. q0 + 31
    const uint64_t win = mz_window(sw, x0 + m - 1);  // bases q0 + m - 1 .. + 31
    // the first m-mer in Horner form, two bases per step
    uint64_t f = 0, rc = 0;
    uint32_t i = 0;
    for (; i + 1 < m; i += 2) f = rol64(f, 2) ^ p2f[(uint32_t)(wout >> (2 * i)) & 15u];
    if (i < m) f = rol64(f, 1) ^ stab[0][(uint32_t)(wout >> (2 * i)) & 3u];
    uint32_t j = m;
    for (; j >= 2; j -= 2) rc = rol64(rc, 2) ^ p2r[(uint32_t)(wout >> (2 * (j - 2))) & 15u];
    if (j == 1) rc = rol64(rc, 1) ^ stab[0][((uint32_t)wout & 3u) ^ 3u];
    sh[mz_pad(q0)] = f <= rc ? f : rc;
#pragma unroll
    for (int j = 1; j < HC; ++j) {
        if ((uint32_t)j < cnt) {
            const uint32_t pr =
                (((uint32_t)(wout >> (2 * (j - 1))) & 3u) << 2) | ((uint32_t)(win >> (2 * j)) & 3u);
            f = rol64(f, 1) ^ tf[pr];
            rc = ror64(rc, 1) ^ tr[pr];
            sh[mz_pad(q0 + j)] = f <= rc ? f : rc;
        }
    }
}

// MODE 0: count the cuts of each tile (tile_count).  MODE 1: write them at
// tile_off.  MODE 2: one pass -- tiles take indices in launch order from
// tile_counter, publish their count in `status` and read their predecessors'
// prefix (decoupled look-back, bounded waits), then write at most `cap`
// entries; the grand total ends in the last tile's status.
// Dynamic shared memory: mz_layout<TT>::bytes.
template <int MODE, int TT = MZ_TT>
__global__ void __launch_bounds__(MZ_THREADS)
    k_minimizers(uint32_t nruns, uint64_t const* __restrict__ tile_start,
                 uint64_t const* __restrict__ soff, uint32_t const* __restrict__ len,
                 uint64_t const* __restrict__ words, uint32_t k, uint32_t m,
                 uint32_t* __restrict__ tile_count, uint64_t const* __restrict__ tile_off,
                 uint64_t* __restrict__ out_min, uint32_t* __restrict__ out_run,
                 uint32_t* __restrict__ out_a, uint32_t* err, uint32_t* tile_counter = nullptr,
                 unsigned long long* status = nullptr, uint64_t ntiles = 0, uint64_t cap = 0) {
    using LY = mz_layout<TT>;
    constexpr int MZ_PER = TT / MZ_THREADS;  // (k-1)-mers per thread
    // m-mers hashed per thread: one chunk each covers the tile and its halo
    constexpr int HC = (LY::HMAX + MZ_THREADS - 1) / MZ_THREADS;
    static_assert(HC <= 32, "a hashing chunk must fit one 32-base window");
    extern __shared__ __align__(16) uint64_t mz_dyn[];
    uint64_t* sw = mz_dyn;                   // staged words (16-byte aligned for the bulk copy)
    uint64_t* sh = mz_dyn + LY::WMAX;        // hashes, then prefix minima (padded index)
    uint64_t* smin = sh + LY::HPAD;          // suffix minima, then window minima
    __shared__ uint64_t stab[4][4];  // rotated ntHash seeds, by base
    __shared__ uint64_t tf[16], tr[16], p2f[16], p2r[16];  // rolling terms by (out base, in base)
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint64_t s_tile, s_excl;

    mz_tables(stab, tf, tr, p2f, p2r, m);
    uint64_t tile = blockIdx.x;
    if (MODE == 2) {
        if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        tile = s_tile;
        if (tile >= ntiles) return;
    }
    // the tile's run: one search by thread 0, shared
    __shared__ uint32_t s_run;
    if (threadIdx.x == 0) s_run = upper_bound_u64(tile_start, nruns + 1, tile) - 1;
    __syncthreads();
    const uint32_t r = s_run;
    const uint64_t t_local = tile - tile_start[r];
    const uint32_t L = len[r];
    const uint32_t W = k - m;
    const uint64_t nk1 = (uint64_t)L - k + 2;  // (k-1)-mers 0..K
    const uint64_t j0 = t_local * TT;
    const uint64_t j1 = (j0 + TT < nk1) ? j0 + TT : nk1;
    const uint64_t e0 = j0 ? j0 - 1 : 0;
    const uint32_t nmin = (uint32_t)(j1 - e0);
    const uint32_t nh = nmin + W - 1;
    // bases [e0, j1 + k - 2) of the run
    const uint64_t pa = soff[r] + e0;
    const uint64_t pb = soff[r] + j1 + k - 2;
    const uint64_t wa = (pa >> 5) & ~uint64_t(1);
    const uint64_t wb = ((pb + 31) >> 5) + 1;
    const uint32_t nw = (uint32_t)(((wb - wa) + 1) & ~uint64_t(1));
    if (!tma_load_1d(sw, words + wa, nw * 8u, &bar, err)) {  // uniform across the block
        if (MODE == 2 && threadIdx.x == 0) atomicExch(&status[tile], (2ull << 62));  // unblock successors
        return;
    }
    const uint32_t rel0 = (uint32_t)(pa - wa * 32);  // stream offset of base e0 in sw
    // canonical m-mer hashes h[0..nh) (h[q] = m-mer at base e0 + q)
    mz_hash<HC>(sw, sh, stab, tf, tr, p2f, p2r, rel0, nh, m);
    __syncthreads();
    // sliding minimum smin[q] = min h[q .. q + W - 1] by segments of W hashes
    // (van Herk / Gil-Werman): with suf[q] the minimum from q to the end of its
    // segment and pre[q] the minimum from its segment's start to q,
    // smin[q] = min(suf[q], pre[q + W - 1]).  One thread per segment writes
    // suf into smin and turns sh into pre in place; then every position takes
    // its minimum.  No data-dependent rescans.
    {
        const uint32_t nseg = (nh + W - 1) / W;
        for (uint32_t g = threadIdx.x; g < nseg; g += MZ_THREADS) {
            const uint32_t a = g * W, e = min(a + W, nh);
            uint64_t run = ~0ull;
            for (uint32_t q = e; q-- > a;) {
                const uint64_t v = sh[mz_pad(q)];
                run = v < run ? v : run;
                if (q < nmin) smin[q] = run;
            }
            run = ~0ull;
            for (uint32_t q = a; q < e; ++q) {
                const uint64_t v = sh[mz_pad(q)];
                run = v < run ? v : run;
                sh[mz_pad(q)] = run;
            }
        }
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nmin; q += MZ_THREADS) {
        const uint64_t a = smin[q], b = sh[mz_pad(q + W - 1)];
        smin[q] = a < b ? a : b;
    }
    __syncthreads();
    // cut points j in [j0, j1): j == 0 or min(j) != min(j - 1).  Position c
    // of the tile is handled in round c / MZ_THREADS by thread c % MZ_THREADS
    // (consecutive threads read consecutive smin words: no bank conflicts);
    // outputs keep position order through per-(round, warp) counts.
    const uint32_t off = (uint32_t)(j0 - e0);  // 0 or 1
    const uint32_t ncut = (uint32_t)(j1 - j0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = MZ_THREADS / 32;
    __shared__ uint32_t wcnt[MZ_PER * NW + 1];
    uint32_t myflags = 0, myrank[MZ_PER];
#pragma unroll
    for (int rr = 0; rr < MZ_PER; ++rr) {
        const uint32_t c = (uint32_t)rr * MZ_THREADS + threadIdx.x;
        bool f = false;
        if (c < ncut) {
            const uint32_t q = c + off;
            f = (j0 + c == 0) || smin[q] != smin[q - 1];
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        myrank[rr] = __popc(bal & lanemask_lt());
        if (f) myflags |= 1u << rr;
        if (lane == 0) wcnt[rr * NW + warp] = __popc(bal);
    }
    __syncthreads();
    // exclusive prefix over (round, warp) in position order, by warp 0
    if (warp == 0) {
        constexpr int E = MZ_PER * NW, PL = (E + 31) / 32;
        uint32_t c[PL], s = 0;
#pragma unroll
        for (int j = 0; j < PL; ++j) {
            const int i = lane * PL + j;
            c[j] = i < E ? wcnt[i] : 0u;
            s += c[j];
        }
        uint32_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        uint32_t ex = x - s;
#pragma unroll
        for (int j = 0; j < PL; ++j) {
            const int i = lane * PL + j;
            if (i < E) wcnt[i] = ex;
            ex += c[j];
        }
        if (lane == 31) wcnt[E] = x;
    }
    __syncthreads();
    const uint32_t tot = wcnt[MZ_PER * NW];
    if (MODE == 0) {
        if (threadIdx.x == 0) tile_count[tile] = tot;
        return;
    }
    uint64_t base;
    if (MODE == 1) {
        base = tile_off[tile];
    } else {
        if (threadIdx.x < 32) {
            uint64_t excl = 0;
            const bool ok = prim::lookback_exclusive(status, tile, tot, excl);
            if (threadIdx.x == 0) {
                if (!ok) set_error(err, ERR_CHAIN_LIMIT);
                s_excl = ok ? excl : ~0ull;
            }
        }
        __syncthreads();
        base = s_excl;
        if (base == ~0ull) return;
    }
#pragma unroll
    for (int rr = 0; rr < MZ_PER; ++rr) {
        if (!((myflags >> rr) & 1u)) continue;
        const uint32_t c = (uint32_t)rr * MZ_THREADS + threadIdx.x;
        const uint64_t o = base + wcnt[rr * NW + warp] + myrank[rr];
        if (MODE == 1 || o < cap) {
            out_min[o] = smin[c + off];
            out_run[o] = r;
            out_a[o] = (uint32_t)(j0 + c);
        }
    }
}

// The one-pass form (MODE 2) for a window known at compile time (W = k - m:
// 19 for k = 31 and 49 for k = 63 with the default m), 4096 (k-1)-mers per
// tile.  After the hashes are staged in shared memory, each thread takes 16
// consecutive (k-1)-mers and finds their window minima in registers: the
// suffix minima of its own 16 hashes, then one running prefix minimum over
// the W - 1 hashes after them, which closes one window per step once it
// reaches past the own 16 (van Herk with the thread's block as the segment).
// The thread also knows the window minimum of the position before its first,
// so it finds its cuts alone; a block scan of the per-thread cut counts and
// the tile look-back place them in order.  No per-position minimum array and
// no stage barriers beyond the hash staging: shared memory is the staged words
// and the hashes only.
constexpr int MZR_C = 16;
constexpr int MZR_TT = MZ_THREADS * MZR_C;
template <int W>
__global__ void __launch_bounds__(MZ_THREADS)
    k_minimizers_reg(uint32_t nruns, uint64_t const* __restrict__ tile_start, uint64_t const* __restrict__ soff,
                     uint32_t const* __restrict__ len, uint64_t const* __restrict__ words, uint32_t k, uint32_t m,
                     uint64_t* __restrict__ out_min, uint32_t* __restrict__ out_run, uint32_t* __restrict__ out_a,
                     uint32_t* err, uint32_t* tile_counter, unsigned long long* status, uint64_t ntiles,
                     uint64_t cap) {
    static_assert(W >= 18 && W <= 62, "window of 18..62 m-mers");
    using LY = mz_layout<MZR_TT>;
    constexpr int HC = (LY::HMAX + MZ_THREADS - 1) / MZ_THREADS;
    extern __shared__ __align__(16) uint64_t mz_dyn[];
    uint64_t* sw = mz_dyn;
    uint64_t* sh = mz_dyn + LY::WMAX;
    __shared__ uint64_t stab[4][4];
    __shared__ uint64_t tf[16], tr[16], p2f[16], p2r[16];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint64_t s_tile, s_excl;
    __shared__ uint32_t s_run;
    __shared__ uint32_t sws[MZ_THREADS / 32 + 1];
    mz_tables(stab, tf, tr, p2f, p2r, m);
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= ntiles) return;
    if (threadIdx.x == 0) s_run = upper_bound_u64(tile_start, nruns + 1, tile) - 1;
    __syncthreads();
    const uint32_t r = s_run;
    const uint64_t t_local = tile - tile_start[r];
    const uint32_t L = len[r];
    const uint64_t nk1 = (uint64_t)L - k + 2;  // (k-1)-mers 0..K
    const uint64_t j0 = t_local * MZR_TT;
    const uint64_t j1 = (j0 + MZR_TT < nk1) ? j0 + MZR_TT : nk1;
    const uint64_t e0 = j0 ? j0 - 1 : 0;
    const uint32_t nmin = (uint32_t)(j1 - e0);
    const uint32_t nh = nmin + W - 1;
    // bases [e0, j1 + k - 2) of the run
    const uint64_t pa = soff[r] + e0;
    const uint64_t pb = soff[r] + j1 + k - 2;
    const uint64_t wa = (pa >> 5) & ~uint64_t(1);
    const uint64_t wb = ((pb + 31) >> 5) + 1;
    const uint32_t nw = (uint32_t)(((wb - wa) + 1) & ~uint64_t(1));
    if (!tma_load_1d(sw, words + wa, nw * 8u, &bar, err)) {  // uniform across the block
        if (threadIdx.x == 0) atomicExch(&status[tile], (2ull << 62));  // unblock successors
        return;
    }
    mz_hash<HC>(sw, sh, stab, tf, tr, p2f, p2r, (uint32_t)(pa - wa * 32), nh, m);
    __syncthreads();
    const uint32_t ncut = (uint32_t)(j1 - j0);
    const uint32_t c0 = threadIdx.x * MZR_C;       // first (k-1)-mer of this thread, from j0
    const uint32_t p0 = (uint32_t)(j0 - e0) + c0;  // its hash index
    uint64_t mn[MZR_C];
    uint32_t mask = 0;
    if (c0 < ncut) {
        uint64_t run = ~0ull;
#pragma unroll
        for (int o = MZR_C - 1; o >= 0; --o) {
            const uint64_t v = sh[mz_pad(p0 + o)];
            run = v < run ? v : run;
            mn[o] = run;
        }
        const uint64_t own = run;  // minimum of the own 16 hashes
        uint64_t P = ~0ull, Pprev = ~0ull;
#pragma unroll
        for (int j = 0; j < W - 1; ++j) {
            const uint64_t v = sh[mz_pad(p0 + MZR_C + j)];
            P = v < P ? v : P;
            if (j == W - 18) Pprev = P;
            if (j >= W - 17) {
                const int o = j - (W - 17);
                mn[o] = mn[o] < P ? mn[o] : P;
            }
        }
        // window [p0 - 1, p0 + W - 2]: the hash before, the own 16, then the
        // first W - 18 hashes after them
        uint64_t prev = ~0ull;
        if (p0 > 0) {
            const uint64_t hb = sh[mz_pad(p0 - 1)];
            prev = hb < own ? hb : own;
            prev = prev < Pprev ? prev : Pprev;
        }
#pragma unroll
        for (int o = 0; o < MZR_C; ++o) {
            const uint32_t c = c0 + o;
            const uint64_t before = o ? mn[o - 1] : prev;
            if (c < ncut && (j0 + c == 0 || mn[o] != before)) mask |= 1u << o;
        }
    }
    uint32_t tot;
    const uint32_t ex = prim::block_exclusive_scan<uint32_t, MZ_THREADS>(__popc(mask), sws, tot);
    if (threadIdx.x < 32) {
        uint64_t excl = 0;
        const bool ok = prim::lookback_exclusive(status, tile, tot, excl);
        if (threadIdx.x == 0) {
            if (!ok) set_error(err, ERR_CHAIN_LIMIT);
            s_excl = ok ? excl : ~0ull;
        }
    }
    __syncthreads();
    const uint64_t base = s_excl;
    if (base == ~0ull) return;
    uint64_t at = base + ex;
#pragma unroll
    for (int o = 0; o < MZR_C; ++o) {
        if ((mask >> o) & 1u) {
            if (at < cap) {
                out_min[at] = mn[o];
                out_run[at] = r;
                out_a[at] = (uint32_t)(j0 + c0 + o);
            }
            ++at;
        }
    }
}

// Dynamic shared memory of a k_minimizers<MODE, TT> launch (opting in above
// the 48 KB default where the tile needs it).
template <int MODE, int TT>
size_t mz_smem() {
    constexpr size_t b = mz_layout<TT>::bytes;
    if (b > 48 * 1024)
        CDBG_CUDA(cudaFuncSetAttribute(k_minimizers<MODE, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b));
    return b;
}

__global__ void k_run_tiles(uint32_t nruns, uint32_t const* __restrict__ len, uint32_t k, uint32_t tt,
                            uint64_t* __restrict__ ntiles) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const uint64_t nk1 = (uint64_t)len[r] - k + 2;
    ntiles[r] = (nk1 + tt - 1) / tt;
}

__global__ void k_run_kmers(uint32_t nruns, uint32_t const* __restrict__ len, uint32_t k,
                            unsigned long long* __restrict__ acc) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = 0, b = 0;
    if (r < nruns) {
        v = (unsigned long long)len[r] - k + 1;
        b = len[r];
    }
    for (int o = 16; o; o >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc, v);
        atomicAdd(acc + 1, b);
    }
}

// Super-k-mer fields from the cut list (bucket_ingester.hpp:80-126).
struct super_fields {
    uint64_t start, key;
    uint32_t len, color, flags, bucket;
};
__device__ __forceinline__ super_fields make_super(uint64_t i, uint64_t n, uint64_t const* __restrict__ minv,
                                                   uint32_t const* __restrict__ run,
                                                   uint32_t const* __restrict__ a_arr,
                                                   uint64_t const* __restrict__ soff,
                                                   uint32_t const* __restrict__ rlen,
                                                   uint32_t const* __restrict__ rcolor,
                                                   uint64_t const* __restrict__ words, uint32_t k, uint32_t B,
                                                   uint32_t bb) {
    super_fields o;
    const uint32_t r = run[i];
    const uint32_t a = a_arr[i];
    const uint64_t K = (uint64_t)rlen[r] - k + 1;
    const bool next_same = (i + 1 < n) && run[i + 1] == r;
    const uint64_t b = next_same ? (uint64_t)a_arr[i + 1] - 1 : K;
    const uint64_t fk = a ? a - 1 : 0;
    const uint64_t lk = b < K - 1 ? b : K - 1;
    o.len = (uint32_t)(lk - fk + k);
    const uint64_t mv = minv[i];
    uint32_t f = 0;
    if (a == 0) f |= 1u;                             // IS_ACGT_BEGIN
    if (!next_same) f |= 2u;                         // IS_ACGT_END
    if (a == 0 || mv < minv[i - 1]) f |= 4u;         // OWNS_FIRST
    if (!next_same || mv < minv[i + 1]) f |= 8u;     // OWNS_LAST
    o.flags = f;
    o.bucket = (uint32_t)((mv >> 1) % B);
    o.start = soff[r] + fk;
    o.color = rcolor[r];
    const uint64_t h = super_hash_dev(words, o.start, o.len);
    o.key = bb ? (((uint64_t)o.bucket << (64 - bb)) | (h >> bb)) : h;
    return o;
}

__global__ void k_super_finalize(uint64_t n, uint64_t const* __restrict__ minv,
                                 uint32_t const* __restrict__ run, uint32_t const* __restrict__ a_arr,
                                 uint64_t const* __restrict__ soff, uint32_t const* __restrict__ rlen,
                                 uint32_t const* __restrict__ rcolor, uint64_t const* __restrict__ words,
                                 uint32_t k, uint32_t B, uint32_t bb, uint64_t* __restrict__ start,
                                 uint32_t* __restrict__ len, uint32_t* __restrict__ color,
                                 uint32_t* __restrict__ flags, uint32_t* __restrict__ bucket,
                                 uint64_t* __restrict__ key) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const super_fields o = make_super(i, n, minv, run, a_arr, soff, rlen, rcolor, words, k, B, bb);
    start[i] = o.start;
    len[i] = o.len;
    color[i] = o.color;
    flags[i] = o.flags;
    bucket[i] = o.bucket;
    key[i] = o.key;
}

// Same fields packed 16 bytes per super-k-mer (start, len, color << 4 |
// flags; colors < 2^28), so the key-order gather of the dedup touches one
// sector per super-k-mer; the bucket is the key's top bits.
__global__ void k_super_finalize_packed(uint64_t n, uint64_t const* __restrict__ minv,
                                        uint32_t const* __restrict__ run, uint32_t const* __restrict__ a_arr,
                                        uint64_t const* __restrict__ soff, uint32_t const* __restrict__ rlen,
                                        uint32_t const* __restrict__ rcolor, uint64_t const* __restrict__ words,
                                        uint32_t k, uint32_t B, uint32_t bb, uint4* __restrict__ packed,
                                        uint64_t* __restrict__ key, uint32_t* err) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const super_fields o = make_super(i, n, minv, run, a_arr, soff, rlen, rcolor, words, k, B, bb);
    if (o.color >> 28) set_error(err, ERR_FIELD_OVERFLOW);
    packed[i] = make_uint4((uint32_t)o.start, (uint32_t)(o.start >> 32), o.len, (o.color << 4) | o.flags);
    key[i] = o.key;
}

__device__ __forceinline__ bool same_bases(uint64_t const* __restrict__ words, uint64_t pa,
                                           uint64_t pb, uint32_t len) {
    for (uint32_t i = 0; i < len; i += 32) {
        uint64_t x = stream_bits64(words, pa + i) ^ stream_bits64(words, pb + i);
        const uint32_t n = len - i;
        if (n < 32) x &= (uint64_t(1) << (2 * n)) - 1;
        if (x) return false;
    }
    return true;
}

// Super-k-mer fields in key order (one gather per field), so the grouping and
// record passes below read them sequentially.
__global__ void k_permute_supers(uint64_t n, uint32_t const* __restrict__ idx, uint64_t const* __restrict__ start,
                                 uint32_t const* __restrict__ len, uint32_t const* __restrict__ color,
                                 uint32_t const* __restrict__ flags, uint64_t* __restrict__ p_start,
                                 uint32_t* __restrict__ p_len, uint32_t* __restrict__ p_color,
                                 uint32_t* __restrict__ p_flags) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t i = idx[p];
    p_start[p] = start[i];
    p_len[p] = len[i];
    p_color[p] = color[i];
    p_flags[p] = flags[i];
}

__global__ void k_permute_packed(uint64_t n, uint32_t const* __restrict__ idx, uint4 const* __restrict__ packed,
                                 uint64_t* __restrict__ p_start, uint32_t* __restrict__ p_len,
                                 uint32_t* __restrict__ p_color, uint32_t* __restrict__ p_flags) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint4 v = packed[idx[p]];
    p_start[p] = ((uint64_t)v.y << 32) | v.x;
    p_len[p] = v.z;
    p_color[p] = v.w >> 4;
    p_flags[p] = v.w & 0xfu;
}

// head[p]: position p starts a new record (key, length or bases differ from
// p - 1); ckeep[p]: p adds a color to its record (the first of each color).
__global__ void k_group_heads_sorted(uint64_t n, uint64_t const* __restrict__ key,
                                     uint64_t const* __restrict__ start, uint32_t const* __restrict__ len,
                                     uint32_t const* __restrict__ color, uint64_t const* __restrict__ words,
                                     uint32_t* __restrict__ head, uint32_t* __restrict__ ckeep) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    bool h = true;
    if (p > 0) {
        h = !(key[p] == key[p - 1] && len[p] == len[p - 1] && same_bases(words, start[p], start[p - 1], len[p]));
        ckeep[p] = (h || color[p] != color[p - 1]) ? 1u : 0u;
    } else {
        ckeep[p] = 1u;
    }
    head[p] = h ? 1u : 0u;
}

__global__ void k_records_fill_sorted(uint64_t n, uint32_t const* __restrict__ head,
                                      uint64_t const* __restrict__ rid_ex, uint32_t const* __restrict__ ckeep,
                                      uint64_t const* __restrict__ cpos, uint64_t const* __restrict__ key,
                                      uint32_t bb, uint64_t const* __restrict__ start,
                                      uint32_t const* __restrict__ len, uint32_t const* __restrict__ color,
                                      uint32_t const* __restrict__ flags, uint64_t* __restrict__ r_start,
                                      uint32_t* __restrict__ r_len, uint32_t* __restrict__ r_flags,
                                      uint64_t* __restrict__ r_coloff, uint32_t* __restrict__ colors,
                                      uint32_t* __restrict__ r_bucket) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint64_t rid = rid_ex[p] + head[p] - 1;  // inclusive count - 1
    if (head[p]) {
        r_start[rid] = start[p];
        r_len[rid] = len[p];
        r_coloff[rid] = cpos[p];
        r_bucket[rid] = bb ? (uint32_t)(key[p] >> (64 - bb)) : 0u;
    }
    const uint32_t f = flags[p];
    if (f != 0xfu) atomicAnd(&r_flags[rid], f);  // AND over the record's copies (starts at 0xf)
    if (ckeep[p]) colors[cpos[p]] = color[p];
}

// bucket_start[b] = first record of bucket b (records are in bucket order):
// each record that starts a bucket fills the starts of the empty buckets
// before it; the last record fills the rest with n.
__global__ void k_bucket_bounds(uint64_t n, uint32_t const* __restrict__ rb, uint32_t B,
                                uint64_t* __restrict__ bucket_start) {
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t b = rb[r];
    const uint32_t prev = r ? rb[r - 1] + 1 : 0;
    for (uint32_t x = prev; x <= b; ++x) bucket_start[x] = r;
    if (r == n - 1)
        for (uint32_t x = b + 1; x <= B; ++x) bucket_start[x] = n;
}

__global__ void k_add_u64(uint64_t* p, uint64_t n, uint64_t v) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] += v;
}

__global__ void k_fill_u32(uint32_t* p, uint64_t n, uint32_t v) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
__global__ void k_iota_u32(uint32_t* p, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (uint32_t)i;
}
__global__ void k_set_last_u64(uint64_t* p, uint64_t idx, uint64_t const* v) { p[idx] = *v; }

// ------------------------------------------------------------ serialization
__device__ __forceinline__ uint32_t varint_len(uint64_t v) {
    uint32_t n = 1;
    while (v >= 0x80) {
        v >>= 7;
        ++n;
    }
    return n;
}
__device__ __forceinline__ uint8_t* varint_put(uint8_t* o, uint64_t v) {
    while (v >= 0x80) {
        *o++ = (uint8_t)((v & 0x7f) | 0x80);
        v >>= 7;
    }
    *o++ = (uint8_t)v;
    return o;
}

__global__ void k_rec_sizes(uint64_t n, uint64_t const* __restrict__ coloff,
                            uint32_t const* __restrict__ colors, uint32_t const* __restrict__ len,
                            uint32_t const* __restrict__ flags, uint64_t* __restrict__ sz) {
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint64_t c0 = coloff[r], c1 = coloff[r + 1];
    uint64_t s = varint_len(c1 - c0);
    uint32_t prev = 0;
    for (uint64_t c = c0; c < c1; ++c) {
        s += varint_len(colors[c] - prev);
        prev = colors[c];
    }
    s += varint_len(((uint64_t)len[r] << 4) | (flags[r] & 0xfu));
    s += (len[r] + 3) / 4;
    sz[r] = s;
}

__global__ void k_rec_write(uint64_t n, uint64_t const* __restrict__ coloff,
                            uint32_t const* __restrict__ colors, uint64_t const* __restrict__ start,
                            uint32_t const* __restrict__ len, uint32_t const* __restrict__ flags,
                            uint64_t const* __restrict__ words, uint64_t const* __restrict__ off,
                            uint8_t* __restrict__ out) {
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint8_t* o = out + off[r];
    const uint64_t c0 = coloff[r], c1 = coloff[r + 1];
    o = varint_put(o, c1 - c0);
    uint32_t prev = 0;
    for (uint64_t c = c0; c < c1; ++c) {
        o = varint_put(o, colors[c] - prev);
        prev = colors[c];
    }
    const uint32_t l = len[r];
    o = varint_put(o, ((uint64_t)l << 4) | (flags[r] & 0xfu));
    const uint64_t st = start[r];
    for (uint32_t i = 0; i < l; i += 32) {
        uint64_t w = stream_bits64(words, st + i);
        const uint32_t nb = (l - i) < 32 ? (l - i) : 32u;
        if (nb < 32) w &= (uint64_t(1) << (2 * nb)) - 1;
        const uint32_t bytes = (nb + 3) / 4;
        for (uint32_t b = 0; b < bytes; ++b) o[b] = (uint8_t)(w >> (8 * b));
        o += bytes;
    }
}

// ------------------------------------------------------------ parsing
__device__ __forceinline__ uint64_t varint_get(uint8_t const* b, uint64_t end, uint64_t& p, bool& ok) {
    uint64_t v = 0;
    uint32_t sh = 0;
    while (p < end) {
        const uint8_t c = b[p++];
        v |= (uint64_t)(c & 0x7f) << sh;
        if (!(c & 0x80)) return v;
        sh += 7;
        if (sh >= 64) break;
    }
    ok = false;
    return v;
}

// One thread per chunk: count records and colors (pass 0) or fill (pass 1).
template <bool FILL>
__global__ void k_parse_chunks(uint8_t const* __restrict__ bytes, uint64_t const* __restrict__ chunk_off,
                               uint32_t nchunks, uint64_t* __restrict__ nrec, uint64_t* __restrict__ ncol,
                               uint64_t const* __restrict__ rec_base, uint64_t const* __restrict__ col_base,
                               uint64_t* __restrict__ r_start, uint32_t* __restrict__ r_len,
                               uint32_t* __restrict__ r_flags, uint64_t* __restrict__ r_coloff,
                               uint32_t* __restrict__ colors, uint32_t* err) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    uint64_t p = chunk_off[c];
    const uint64_t end = chunk_off[c + 1];
    uint64_t nr = 0, nc = 0;
    uint64_t ro = FILL ? rec_base[c] : 0, co = FILL ? col_base[c] : 0;
    while (p < end) {
        bool ok = true;
        const uint64_t k = varint_get(bytes, end, p, ok);
        if (FILL) r_coloff[ro + nr] = co + nc;
        uint32_t prev = 0;
        for (uint64_t i = 0; i < k && ok; ++i) {
            prev += (uint32_t)varint_get(bytes, end, p, ok);
            if (FILL) colors[co + nc + i] = prev;
        }
        const uint64_t lf = varint_get(bytes, end, p, ok);
        const uint64_t l = lf >> 4;
        const uint64_t nb = (l + 3) / 4;
        if (!ok || p + nb > end || l >= (1ull << 32)) {
            set_error(err, ERR_BAD_RECORD);
            return;
        }
        if (FILL) {
            r_start[ro + nr] = p * 4;  // byte offset -> 2-bit stream position
            r_len[ro + nr] = (uint32_t)l;
            r_flags[ro + nr] = (uint32_t)(lf & 0xf);
        }
        p += nb;
        nc += k;
        ++nr;
    }
    if (!FILL) {
        nrec[c] = nr;
        ncol[c] = nc;
    }
}

__global__ void k_bucket_bytes(uint32_t B, uint64_t const* __restrict__ bstart,
                               uint64_t const* __restrict__ rec_off, uint64_t* __restrict__ boff) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b <= B) boff[b] = rec_off[bstart[b]];
}

__global__ void k_chunk_bucket_counts(uint32_t nchunks, uint32_t const* __restrict__ chunk_bucket,
                                      uint64_t const* __restrict__ nrec,
                                      unsigned long long* __restrict__ bcnt) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nchunks) atomicAdd(&bcnt[chunk_bucket[c]], (unsigned long long)nrec[c]);
}

inline unsigned grid(uint64_t n, unsigned t) { return (unsigned)ceil_div(n, t); }

template <typename T>
T read_dev(T const* p, cudaStream_t st) {
    T v;
    read_small(&v, p, sizeof(T), st);
    return v;
}

}  // namespace

// ----------------------------------------------------------------- host side
void build_runs(seq_input const& in, uint32_t k, dev_arena& A, cudaStream_t st, run_table& rt,
                dev_arena& out, uint64_t* words_out, uint64_t word_base, uint64_t words_cap) {
    rt = run_table();
    const uint64_t npos = in.nbytes + 1;
    const uint64_t tiles = ceil_div(npos, EV_TILE);
    uint32_t* tcount = A.alloc<uint32_t>(tiles);
    uint64_t* toff = A.alloc<uint64_t>(tiles + 1);
    // bit p of `starts`: a sequence starts at p (or p = nbytes)
    const uint64_t nsw = (in.nbytes >> 5) + 2;
    uint32_t* starts = A.alloc<uint32_t>(nsw);
    CDBG_CUDA(cudaMemsetAsync(starts, 0, 4 * nsw, st));
    k_seq_starts<<<grid((uint64_t)in.num_seqs + 1, 256), 256, 0, st>>>(in.seq_off, in.num_seqs, starts);
    CDBG_CHECK_LAUNCH();
    // one pass into room for a run every 64 bases (two events each); input
    // with more runs than that takes the two passes
    uint64_t ev_cap = in.nbytes / 32 + 1024;
    uint64_t* ev = A.alloc<uint64_t>(ev_cap);
    uint64_t nev = 0;
    {
        uint32_t* counter = A.alloc<uint32_t>(1);
        unsigned long long* status = A.alloc<unsigned long long>(tiles);
        unsigned long long* total = A.alloc<unsigned long long>(1);
        uint32_t* lerr = A.alloc<uint32_t>(1);
        CDBG_CUDA(cudaMemsetAsync(counter, 0, 4, st));
        CDBG_CUDA(cudaMemsetAsync(status, 0, 8 * tiles, st));
        CDBG_CUDA(cudaMemsetAsync(lerr, 0, 4, st));
        {
            CDBG_PROF("k_run_events", st);
            k_run_events_1p<<<(unsigned)tiles, EV_THREADS, 0, st>>>(in.ascii, in.nbytes, starts, tiles, counter,
                                                                   status, ev, ev_cap, total, lerr);
        }
        CDBG_CHECK_LAUNCH();
        uint64_t got[2] = {0, 0};
        read_small(&got[0], total, 8, st);
        uint32_t le = 0;
        read_small(&le, lerr, 4, st);
        if (le) throw std::runtime_error("run events: look-back wait limit reached");
        nev = got[0];
    }
    if (nev > ev_cap) {
        {
            CDBG_PROF("k_run_events", st);
            k_run_events<false><<<(unsigned)tiles, EV_THREADS, 0, st>>>(in.ascii, in.nbytes, starts, tcount,
                                                                         nullptr, nullptr);
        }
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(tcount, toff, tiles, A, st, toff + tiles);
        nev = read_dev(toff + tiles, st);
        ev = A.alloc<uint64_t>(nev);
        {
            CDBG_PROF("k_run_events", st);
            k_run_events<true><<<(unsigned)tiles, EV_THREADS, 0, st>>>(in.ascii, in.nbytes, starts, tcount, toff,
                                                                        ev);
        }
        CDBG_CHECK_LAUNCH();
    }
    const uint64_t nraw = nev / 2;
    if (nraw == 0) return;
    uint64_t* src = A.alloc<uint64_t>(nraw);
    uint32_t* len = A.alloc<uint32_t>(nraw);
    uint32_t* color = A.alloc<uint32_t>(nraw);
    uint32_t* keep = A.alloc<uint32_t>(nraw);
    uint64_t* kpos = A.alloc<uint64_t>(nraw + 1);
    uint32_t* err = A.alloc<uint32_t>(1);
    CDBG_CUDA(cudaMemsetAsync(err, 0, 4, st));
    k_runs_from_events<<<grid(nraw, 256), 256, 0, st>>>(ev, nraw, in.seq_off, in.num_seqs,
                                                         in.seq_color, k, src, len, color, keep, err);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint32_t, uint64_t>(keep, kpos, nraw, A, st, kpos + nraw);
    const uint64_t nruns = read_dev(kpos + nraw, st);
    if (read_dev(err, st) != 0) throw std::runtime_error("run length exceeds 2^32 bases");
    if (nruns == 0) return;
    if (nruns >= 0xffffffffull) throw std::runtime_error("too many ACGT runs");
    rt.n = (uint32_t)nruns;
    rt.src = A.alloc<uint64_t>(nruns);
    rt.len = A.alloc<uint32_t>(nruns);
    rt.color = A.alloc<uint32_t>(nruns);
    uint64_t* padded = A.alloc<uint64_t>(nruns);
    rt.soff = A.alloc<uint64_t>(nruns + 1);
    k_runs_compact<<<grid(nraw, 256), 256, 0, st>>>(nraw, keep, kpos, src, len, color, rt.src, rt.len,
                                                     rt.color, padded);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint64_t, uint64_t>(padded, rt.soff, nruns, A, st, rt.soff + nruns);
    const uint64_t total = read_dev(rt.soff + nruns, st);
    const uint64_t nwd = total / 32;
    uint64_t* dst;
    if (words_out) {
        // this batch's runs go at word `word_base` of a shared stream
        if (word_base + nwd + 8 > words_cap) throw std::runtime_error("2-bit stream capacity exceeded");
        rt.words = words_out;
        rt.nwords = word_base + nwd + 8;
        dst = words_out + word_base;
    } else {
        rt.nwords = nwd + 8;
        rt.words = out.alloc<uint64_t>(rt.nwords);
        dst = rt.words;
    }
    CDBG_CUDA(cudaMemsetAsync(dst + nwd, 0, 8 * 8, st));
    if (nwd) {
        {
            CDBG_PROF("k_pack", st);
            k_pack<<<grid(nwd, 256), 256, 0, st>>>(in.ascii, rt.n, rt.soff, rt.src, rt.len, nwd, dst);
        }
        CDBG_CHECK_LAUNCH();
    }
    if (words_out && word_base) {
        k_add_u64<<<grid(nruns + 1, 256), 256, 0, st>>>(rt.soff, nruns + 1, word_base * 32);
        CDBG_CHECK_LAUNCH();
    }
    unsigned long long* acc = A.alloc<unsigned long long>(2);
    CDBG_CUDA(cudaMemsetAsync(acc, 0, 16, st));
    k_run_kmers<<<grid(nruns, 256), 256, 0, st>>>(rt.n, rt.len, k, acc);
    CDBG_CHECK_LAUNCH();
    unsigned long long h[2];
    read_small(h, acc, 16, st);
    rt.n_kmers = h[0];
    rt.n_bases = h[1];
}

template <int TT>
void find_supers_tt(run_table const& rt, uint32_t k, uint32_t m, uint32_t B, dev_arena& A,
                    cudaStream_t st, super_list& out, uint32_t* d_err, bool packed);

void find_supers(run_table const& rt, uint32_t k, uint32_t m, uint32_t B, dev_arena& A,
                 cudaStream_t st, super_list& out, uint32_t* d_err, uint32_t tile, bool packed) {
    if (tile == 1024)
        find_supers_tt<1024>(rt, k, m, B, A, st, out, d_err, packed);
    else if (tile == 2048)
        find_supers_tt<2048>(rt, k, m, B, A, st, out, d_err, packed);
    else if (tile == 4096 || tile == 0)
        find_supers_tt<4096>(rt, k, m, B, A, st, out, d_err, packed);
    else
        throw std::runtime_error("minimizer tile must be 1024, 2048 or 4096");
}

template <int TT>
void find_supers_tt(run_table const& rt, uint32_t k, uint32_t m, uint32_t B, dev_arena& A,
                    cudaStream_t st, super_list& out, uint32_t* d_err, bool packed) {
    out = super_list();
    if (rt.n == 0) return;
    if (k < 2 || m >= k || k - m > 62 || m > 32)
        throw std::runtime_error("unsupported k/m combination");
    uint64_t* ntl = A.alloc<uint64_t>(rt.n);
    uint64_t* tstart = A.alloc<uint64_t>(rt.n + 1);
    k_run_tiles<<<grid(rt.n, 256), 256, 0, st>>>(rt.n, rt.len, k, TT, ntl);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint64_t, uint64_t>(ntl, tstart, rt.n, A, st, tstart + rt.n);
    const uint64_t ntiles = read_dev(tstart + rt.n, st);
    // one pass with a capacity of 1/4 of the (k-1)-mers (about 2.5x the
    // density of random sequence); the exact two-pass path if it overflows
    const uint64_t npos = rt.n_kmers + rt.n;
    uint64_t cap = std::max<uint64_t>(1ull << 20, npos / 4);
    uint64_t* minv = A.alloc<uint64_t>(cap);
    uint32_t* run = A.alloc<uint32_t>(cap);
    uint32_t* aa = A.alloc<uint32_t>(cap);
    unsigned long long* status = A.alloc<unsigned long long>(ntiles);
    uint32_t* counter = A.alloc<uint32_t>(1);
    CDBG_CUDA(cudaMemsetAsync(status, 0, 8 * ntiles, st));
    CDBG_CUDA(cudaMemsetAsync(counter, 0, 4, st));
    {
        CDBG_PROF("k_minimizers", st);
        // the register-window form for the two windows of the default m
        // (k = 31 and k = 63); the shared-memory form otherwise
        constexpr size_t reg_smem = sizeof(uint64_t) * (mz_layout<MZR_TT>::WMAX + mz_layout<MZR_TT>::HPAD);
        if (TT == MZR_TT && k - m == 19)
            k_minimizers_reg<19><<<(unsigned)ntiles, MZ_THREADS, reg_smem, st>>>(
                rt.n, tstart, rt.soff, rt.len, rt.words, k, m, minv, run, aa, d_err, counter, status, ntiles, cap);
        else if (TT == MZR_TT && k - m == 49)
            k_minimizers_reg<49><<<(unsigned)ntiles, MZ_THREADS, reg_smem, st>>>(
                rt.n, tstart, rt.soff, rt.len, rt.words, k, m, minv, run, aa, d_err, counter, status, ntiles, cap);
        else
            k_minimizers<2, TT><<<(unsigned)ntiles, MZ_THREADS, mz_smem<2, TT>(), st>>>(
                rt.n, tstart, rt.soff, rt.len, rt.words, k, m, nullptr, nullptr, minv, run, aa, d_err, counter,
                status, ntiles, cap);
    }
    CDBG_CHECK_LAUNCH();
    uint64_t n = read_dev(status + ntiles - 1, st) & ((1ull << 62) - 1);
    if (n > cap) {
        uint32_t* tcount = A.alloc<uint32_t>(ntiles);
        uint64_t* toff = A.alloc<uint64_t>(ntiles + 1);
        {
            CDBG_PROF("k_minimizers", st);
            k_minimizers<0, TT><<<(unsigned)ntiles, MZ_THREADS, mz_smem<0, TT>(), st>>>(
                rt.n, tstart, rt.soff, rt.len, rt.words, k, m, tcount, nullptr, nullptr, nullptr, nullptr, d_err);
        }
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(tcount, toff, ntiles, A, st, toff + ntiles);
        n = read_dev(toff + ntiles, st);
        minv = A.alloc<uint64_t>(n);
        run = A.alloc<uint32_t>(n);
        aa = A.alloc<uint32_t>(n);
        {
            CDBG_PROF("k_minimizers", st);
            k_minimizers<1, TT><<<(unsigned)ntiles, MZ_THREADS, mz_smem<1, TT>(), st>>>(
                rt.n, tstart, rt.soff, rt.len, rt.words, k, m, tcount, toff, minv, run, aa, d_err);
        }
        CDBG_CHECK_LAUNCH();
    }
    if (n >= 0xffffffffull) throw std::runtime_error("more than 2^32 super-k-mers in one call");
    out.n = n;
    out.key = A.alloc<uint64_t>(n);
    uint32_t bb = 0;
    while ((1ull << bb) < B) ++bb;
    if (packed) {
        out.packed = A.alloc<uint4>(n);
        CDBG_PROF("k_super_finalize", st);
        k_super_finalize_packed<<<grid(n, 256), 256, 0, st>>>(n, minv, run, aa, rt.soff, rt.len, rt.color, rt.words,
                                                               k, B, bb, out.packed, out.key, d_err);
    } else {
        out.start = A.alloc<uint64_t>(n);
        out.len = A.alloc<uint32_t>(n);
        out.color = A.alloc<uint32_t>(n);
        out.flags = A.alloc<uint32_t>(n);
        out.bucket = A.alloc<uint32_t>(n);
        CDBG_PROF("k_super_finalize", st);
        k_super_finalize<<<grid(n, 256), 256, 0, st>>>(n, minv, run, aa, rt.soff, rt.len, rt.color, rt.words,
                                                        k, B, bb, out.start, out.len, out.color, out.flags,
                                                        out.bucket, out.key);
    }
    CDBG_CHECK_LAUNCH();
}

namespace {
__device__ __forceinline__ uint32_t key_bucket(uint64_t key, uint32_t bb) {
    return bb ? (uint32_t)(key >> (64 - bb)) : 0u;
}
__global__ void k_range_flags(uint64_t n, uint64_t const* __restrict__ key, uint32_t bb, uint32_t lo, uint32_t hi,
                              uint32_t* __restrict__ keep) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = key_bucket(key[i], bb);
    keep[i] = (b >= lo && b < hi) ? 1u : 0u;
}
template <typename T>
__global__ void k_compact(uint64_t n, uint32_t const* __restrict__ keep, uint64_t const* __restrict__ pos,
                          T const* __restrict__ in, T* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && keep[i]) out[pos[i]] = in[i];
}
}  // namespace

void keep_bucket_range(super_list& sl, uint32_t B, uint32_t lo, uint32_t hi, dev_arena& A, cudaStream_t st) {
    if (lo == 0 && hi >= B) return;
    const uint64_t n = sl.n;
    if (n == 0) return;
    uint32_t bb = 0;
    while ((1ull << bb) < B) ++bb;
    uint32_t* keep = A.alloc<uint32_t>(n);
    uint64_t* pos = A.alloc<uint64_t>(n + 1);
    k_range_flags<<<grid(n, 256), 256, 0, st>>>(n, sl.key, bb, lo, hi, keep);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint32_t, uint64_t>(keep, pos, n, A, st, pos + n);
    const uint64_t m = read_dev(pos + n, st);
    super_list o = sl;
    o.n = m;
    auto pack = [&](auto* in, auto*& out) {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(in)>>;
        if (!in) return;
        T* dst = A.alloc<T>(m + 1);
        k_compact<T><<<grid(n, 256), 256, 0, st>>>(n, keep, pos, in, dst);
        CDBG_CHECK_LAUNCH();
        out = dst;
    };
    pack(sl.key, o.key);
    pack(sl.packed, o.packed);
    pack(sl.start, o.start);
    pack(sl.len, o.len);
    pack(sl.color, o.color);
    pack(sl.flags, o.flags);
    pack(sl.bucket, o.bucket);
    sl = o;
}

void build_records(run_table const& rt, super_list& sl, uint32_t k, uint32_t B, dev_arena& A,
                   cudaStream_t st, record_set& rs, uint32_t* d_err, dev_arena& out) {
    (void)k;
    (void)d_err;
    rs = record_set();
    rs.B = B;
    rs.words = rt.words;
    rs.nwords = rt.nwords;
    rs.n_occ_supers = sl.n;
    rs.bucket_start = out.alloc<uint64_t>(B + 1);
    const uint64_t n = sl.n;
    if (n == 0) {
        CDBG_CUDA(cudaMemsetAsync(rs.bucket_start, 0, 8 * (B + 1), st));
        rs.col_off = out.alloc<uint64_t>(1);
        CDBG_CUDA(cudaMemsetAsync(rs.col_off, 0, 8, st));
        return;
    }
    uint32_t* idx = A.alloc<uint32_t>(n);
    k_iota_u32<<<grid(n, 256), 256, 0, st>>>(idx, n);
    CDBG_CHECK_LAUNCH();
    // sort a copy of the keys (the super list keeps its input order)
    uint64_t* skey = A.alloc<uint64_t>(n);
    CDBG_CUDA(cudaMemcpyAsync(skey, sl.key, n * 8, cudaMemcpyDeviceToDevice, st));
    prim::sort_pairs_u64_exact<uint32_t>(skey, idx, n, A, st, d_err);
    uint64_t* p_start = A.alloc<uint64_t>(n);
    uint32_t* p_len = A.alloc<uint32_t>(n);
    uint32_t* p_color = A.alloc<uint32_t>(n);
    uint32_t* p_flags = A.alloc<uint32_t>(n);
    {
        CDBG_PROF("k_permute_supers", st);
        if (sl.packed)
            k_permute_packed<<<grid(n, 256), 256, 0, st>>>(n, idx, sl.packed, p_start, p_len, p_color, p_flags);
        else
            k_permute_supers<<<grid(n, 256), 256, 0, st>>>(n, idx, sl.start, sl.len, sl.color, sl.flags, p_start,
                                                            p_len, p_color, p_flags);
    }
    CDBG_CHECK_LAUNCH();
    uint32_t* head = A.alloc<uint32_t>(n);
    uint32_t* ckeep = A.alloc<uint32_t>(n);
    {
        CDBG_PROF("k_group_heads", st);
        k_group_heads_sorted<<<grid(n, 256), 256, 0, st>>>(n, skey, p_start, p_len, p_color, rt.words, head, ckeep);
    }
    CDBG_CHECK_LAUNCH();
    uint64_t* rid = A.alloc<uint64_t>(n + 1);
    uint64_t* cpos = A.alloc<uint64_t>(n + 1);
    prim::exclusive_scan<uint32_t, uint64_t>(head, rid, n, A, st, rid + n);
    prim::exclusive_scan<uint32_t, uint64_t>(ckeep, cpos, n, A, st, cpos + n);
    uint64_t tot[2];
    read_small(&tot[0], rid + n, 8, st);
    read_small(&tot[1], cpos + n, 8, st);
    const uint64_t nr = tot[0], nc = tot[1];
    rs.n = nr;
    rs.ncolors = nc;
    rs.start = out.alloc<uint64_t>(nr);
    rs.len = out.alloc<uint32_t>(nr);
    rs.flags = out.alloc<uint32_t>(nr);
    rs.col_off = out.alloc<uint64_t>(nr + 1);
    rs.colors = out.alloc<uint32_t>(nc);
    uint32_t* rb = A.alloc<uint32_t>(nr);
    k_fill_u32<<<grid(nr, 256), 256, 0, st>>>(rs.flags, nr, 0xfu);
    CDBG_CHECK_LAUNCH();
    uint32_t bb = 0;
    while ((1ull << bb) < B) ++bb;
    {
        CDBG_PROF("k_records_fill", st);
        k_records_fill_sorted<<<grid(n, 256), 256, 0, st>>>(n, head, rid, ckeep, cpos, skey, bb, p_start, p_len,
                                                             p_color, p_flags, rs.start, rs.len, rs.flags,
                                                             rs.col_off, rs.colors, rb);
    }
    CDBG_CHECK_LAUNCH();
    k_set_last_u64<<<1, 1, 0, st>>>(rs.col_off, nr, cpos + n);
    CDBG_CHECK_LAUNCH();
    k_bucket_bounds<<<grid(nr, 256), 256, 0, st>>>(nr, rb, B, rs.bucket_start);
    CDBG_CHECK_LAUNCH();
}

// Serialized size of every record summed into *sum (the uncompressed bytes
// the bucket files would hold); same per-record arithmetic as k_rec_sizes.
__global__ void k_rec_bytes_sum(uint64_t n, uint64_t const* __restrict__ coloff,
                                uint32_t const* __restrict__ colors, uint32_t const* __restrict__ len,
                                uint32_t const* __restrict__ flags, unsigned long long* __restrict__ sum) {
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long s = 0;
    if (r < n) {
        const uint64_t c0 = coloff[r], c1 = coloff[r + 1];
        s = varint_len(c1 - c0);
        uint32_t prev = 0;
        for (uint64_t c = c0; c < c1; ++c) {
            s += varint_len(colors[c] - prev);
            prev = colors[c];
        }
        s += varint_len(((uint64_t)len[r] << 4) | (flags[r] & 0xfu));
        s += (len[r] + 3) / 4;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(sum, s);
}

void record_bytes_async(record_set const& rs, unsigned long long* d_sum, cudaStream_t st) {
    CDBG_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(unsigned long long), st));
    if (rs.n == 0) return;
    {
        CDBG_PROF("k_rec_bytes_sum", st);
        k_rec_bytes_sum<<<grid(rs.n, 256), 256, 0, st>>>(rs.n, rs.col_off, rs.colors, rs.len, rs.flags, d_sum);
    }
    CDBG_CHECK_LAUNCH();
}

void serialize_records(record_set const& rs, dev_arena& A, cudaStream_t st, serialized_buckets& out) {
    out = serialized_buckets();
    out.rec_off = A.alloc<uint64_t>(rs.n + 1);
    out.bucket_off = A.alloc<uint64_t>(rs.B + 1);
    if (rs.n == 0) {
        CDBG_CUDA(cudaMemsetAsync(out.rec_off, 0, 8, st));
        CDBG_CUDA(cudaMemsetAsync(out.bucket_off, 0, 8ull * (rs.B + 1), st));
        out.bytes = A.alloc<uint8_t>(16);
        return;
    }
    uint64_t* sz = A.alloc<uint64_t>(rs.n);
    {
        CDBG_PROF("k_rec_sizes", st);
        k_rec_sizes<<<grid(rs.n, 256), 256, 0, st>>>(rs.n, rs.col_off, rs.colors, rs.len, rs.flags, sz);
    }
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint64_t, uint64_t>(sz, out.rec_off, rs.n, A, st, out.rec_off + rs.n);
    out.nbytes = read_dev(out.rec_off + rs.n, st);
    out.bytes = A.alloc<uint8_t>(out.nbytes + 16);
    {
        CDBG_PROF("k_rec_write", st);
        k_rec_write<<<grid(rs.n, 256), 256, 0, st>>>(rs.n, rs.col_off, rs.colors, rs.start, rs.len, rs.flags,
                                                      rs.words, out.rec_off, out.bytes);
    }
    CDBG_CHECK_LAUNCH();
    k_bucket_bytes<<<grid(rs.B + 1, 256), 256, 0, st>>>(rs.B, rs.bucket_start, out.rec_off, out.bucket_off);
    CDBG_CHECK_LAUNCH();
}

void parse_records(uint8_t const* bytes, uint64_t nbytes, uint64_t const* chunk_off,
                   uint32_t const* chunk_bucket, uint32_t nchunks, uint32_t B, dev_arena& A,
                   cudaStream_t st, record_set& rs, uint32_t* d_err) {
    (void)nbytes;
    rs = record_set();
    rs.B = B;
    rs.words = reinterpret_cast<uint64_t const*>(bytes);
    rs.nwords = (nbytes + 7) / 8;
    rs.bucket_start = A.alloc<uint64_t>(B + 1);
    uint64_t* nrec = A.alloc<uint64_t>(nchunks + 1);
    uint64_t* ncol = A.alloc<uint64_t>(nchunks + 1);
    uint64_t* rbase = A.alloc<uint64_t>(nchunks + 1);
    uint64_t* cbase = A.alloc<uint64_t>(nchunks + 1);
    if (nchunks) {
        k_parse_chunks<false><<<grid(nchunks, 64), 64, 0, st>>>(bytes, chunk_off, nchunks, nrec, ncol,
                                                                 nullptr, nullptr, nullptr, nullptr,
                                                                 nullptr, nullptr, nullptr, d_err);
        CDBG_CHECK_LAUNCH();
    }
    prim::exclusive_scan<uint64_t, uint64_t>(nrec, rbase, nchunks, A, st, rbase + nchunks);
    prim::exclusive_scan<uint64_t, uint64_t>(ncol, cbase, nchunks, A, st, cbase + nchunks);
    uint64_t t[2];
    CDBG_CUDA(cudaMemcpyAsync(&t[0], rbase + nchunks, 8, cudaMemcpyDeviceToHost, st));
    CDBG_CUDA(cudaMemcpyAsync(&t[1], cbase + nchunks, 8, cudaMemcpyDeviceToHost, st));
    CDBG_CUDA(cudaStreamSynchronize(st));
    rs.n = t[0];
    rs.ncolors = t[1];
    rs.start = A.alloc<uint64_t>(rs.n);
    rs.len = A.alloc<uint32_t>(rs.n);
    rs.flags = A.alloc<uint32_t>(rs.n);
    rs.col_off = A.alloc<uint64_t>(rs.n + 1);
    rs.colors = A.alloc<uint32_t>(rs.ncolors);
    if (nchunks) {
        k_parse_chunks<true><<<grid(nchunks, 64), 64, 0, st>>>(bytes, chunk_off, nchunks, nrec, ncol, rbase,
                                                                cbase, rs.start, rs.len, rs.flags,
                                                                rs.col_off, rs.colors, d_err);
        CDBG_CHECK_LAUNCH();
    }
    k_set_last_u64<<<1, 1, 0, st>>>(rs.col_off, rs.n, cbase + nchunks);
    CDBG_CHECK_LAUNCH();
    unsigned long long* bc = A.alloc<unsigned long long>(B);
    CDBG_CUDA(cudaMemsetAsync(bc, 0, 8ull * B, st));
    if (nchunks) {
        k_chunk_bucket_counts<<<grid(nchunks, 256), 256, 0, st>>>(nchunks, chunk_bucket, nrec, bc);
        CDBG_CHECK_LAUNCH();
    }
    prim::exclusive_scan<unsigned long long, uint64_t>(bc, rs.bucket_start, B, A, st, rs.bucket_start + B);
}

}  // namespace cdbg

namespace cdbg {

// ===========================================================================
// Super-k-mer finder for callers that cannot allocate device memory.
//
// Some callers run where they may not call cudaMalloc / cudaFree or anything
// that allocates on the device: code that must not add memory of its own next
// to a host application's pool (a framework's caching allocator, a memory
// budget managed elsewhere), or code running with allocation forbidden. They
// pre-pack their ACGT runs into device memory and hand in output arrays; this
// entry point finds the super-k-mers of those runs using only the fixed
// scratch below, which every GPU that loads this library holds until the
// process exits.
//
// Limit: at most NOALLOC_MAX_TILES tiles per call, a run taking
// ceil((len - k + 2) / 2048) tiles -- at most 512 runs and 1,048,576
// (k-1)-mers per call.  Larger inputs are rejected; split them.
// All calls share the scratch and it keeps the previous call's contents:
// calls that overlap on the GPU (other streams, other host threads) race.
// ===========================================================================

namespace {

constexpr uint32_t NOALLOC_MAX_TILES = 512;
constexpr uint64_t NOALLOC_MAX_SUPERS = (uint64_t)NOALLOC_MAX_TILES * MZ_TT;

struct noalloc_scratch {
    uint64_t run_tiles[NOALLOC_MAX_TILES];
    uint64_t tile_start[NOALLOC_MAX_TILES + 1];
    uint32_t tile_count[NOALLOC_MAX_TILES];
    uint64_t tile_off[NOALLOC_MAX_TILES + 1];
    uint64_t minv[NOALLOC_MAX_SUPERS];
    uint32_t run[NOALLOC_MAX_SUPERS];
    uint32_t a[NOALLOC_MAX_SUPERS];
    uint64_t key[NOALLOC_MAX_SUPERS];
    uint32_t err;
};

// The scratch itself (about 24 MiB).  Host code must not pass this name to a
// kernel: on the host it is only a stand-in; its device address comes from
// cudaGetSymbolAddress (noalloc_scratch_ptr below).
static __device__ __align__(256) noalloc_scratch g_noalloc_scratch;

// Tiles per run like k_run_tiles, for caller-supplied runs: a run shorter
// than k has no k-mer and would make the tile arithmetic wrap, so it counts
// zero tiles and sets `err` (the host reads it before any tile kernel runs).
__global__ void k_noalloc_run_tiles(uint32_t nruns, uint32_t const* __restrict__ len, uint32_t k, uint32_t tt,
                                    uint64_t* __restrict__ ntiles, uint32_t* err) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const uint32_t L = len[r];
    if (L < k) {
        set_error(err, ERR_BAD_RECORD);
        ntiles[r] = 0;
        return;
    }
    ntiles[r] = ((uint64_t)L - k + 2 + tt - 1) / tt;
}

// Exclusive scan of n <= NOALLOC_MAX_TILES values by one block; the total goes
// to out[n].
template <typename T>
__global__ void __launch_bounds__(1024) k_noalloc_scan(T const* __restrict__ in, uint32_t n,
                                                       uint64_t* __restrict__ out) {
    __shared__ uint64_t sw[1024 / 32 + 1];
    const uint64_t v = threadIdx.x < n ? (uint64_t)in[threadIdx.x] : 0;
    uint64_t tot;
    const uint64_t ex = prim::block_exclusive_scan<uint64_t, 1024>(v, sw, tot);
    if (threadIdx.x < n) out[threadIdx.x] = ex;
    if (threadIdx.x == 0) out[n] = tot;
}

std::mutex g_noalloc_mu;
noalloc_scratch* g_noalloc_ptr[256] = {};

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does this; make that first call before
// any stream capture).  The address stays cached for the life of the process,
// so it is stale after the caller resets the device (cudaDeviceReset).
noalloc_scratch* noalloc_scratch_ptr() {
    int dev = 0;
    CDBG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) throw std::runtime_error("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw std::runtime_error(std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<noalloc_scratch*>(p);
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

}  // namespace cdbg

extern "C" int cdbg_gpu_supers_noalloc(const uint64_t* words, const uint64_t* run_soff,
                                       const uint32_t* run_len, const uint32_t* run_color,
                                       uint32_t num_runs, uint32_t k, uint32_t m, uint32_t num_buckets,
                                       uint64_t* out_start, uint32_t* out_len, uint32_t* out_color,
                                       uint32_t* out_flags, uint32_t* out_bucket, uint64_t out_cap,
                                       uint64_t* n_supers, void* stream) {
    using namespace cdbg;
    try {
        if (n_supers) *n_supers = 0;
        if (k < 2 || k > 63 || m == 0 || m >= k || m > 32 || k - m > 62)
            throw std::runtime_error("unsupported k/m combination");
        if (num_buckets == 0) throw std::runtime_error("num_buckets must be > 0");
        if (num_runs > NOALLOC_MAX_TILES)
            throw std::runtime_error("more than 512 runs in one call (each run needs at least one tile)");
        // the tile kernel stages words from `words` with bulk copies, which
        // need 16-byte aligned global addresses
        if (reinterpret_cast<uintptr_t>(words) & 15u)
            throw std::runtime_error("words must be 16-byte aligned");
        cudaStream_t st = (cudaStream_t)stream;
        noalloc_scratch* s = noalloc_scratch_ptr();
        CDBG_CUDA(cudaMemsetAsync(&s->err, 0, sizeof(uint32_t), st));
        if (num_runs == 0) return 0;
        k_noalloc_run_tiles<<<grid(num_runs, 256), 256, 0, st>>>(num_runs, run_len, k, MZ_TT, s->run_tiles,
                                                                 &s->err);
        CDBG_CHECK_LAUNCH();
        k_noalloc_scan<uint64_t><<<1, 1024, 0, st>>>(s->run_tiles, num_runs, s->tile_start);
        CDBG_CHECK_LAUNCH();
        struct {
            uint64_t v;
            uint32_t err;
        } rb{0, 0};
        CDBG_CUDA(cudaMemcpyAsync(&rb.v, &s->tile_start[num_runs], 8, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaMemcpyAsync(&rb.err, &s->err, 4, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        if (rb.err) throw std::runtime_error("a run is shorter than k bases");
        const uint64_t ntiles = rb.v;
        if (ntiles > NOALLOC_MAX_TILES)
            throw std::runtime_error("input needs " + std::to_string(ntiles) +
                                     " tiles; at most 512 tiles of 2048 (k-1)-mers per call");
        // a tile that gives up (bounded staging wait) writes no count: start
        // from zero rather than the previous call's counts
        CDBG_CUDA(cudaMemsetAsync(s->tile_count, 0, sizeof(uint32_t) * ntiles, st));
        k_minimizers<0><<<(unsigned)ntiles, MZ_THREADS, mz_smem<0, MZ_TT>(), st>>>(num_runs, s->tile_start, run_soff, run_len,
                                                                 words, k, m, s->tile_count, nullptr, nullptr,
                                                                 nullptr, nullptr, &s->err);
        CDBG_CHECK_LAUNCH();
        k_noalloc_scan<uint32_t><<<1, 1024, 0, st>>>(s->tile_count, (uint32_t)ntiles, s->tile_off);
        CDBG_CHECK_LAUNCH();
        CDBG_CUDA(cudaMemcpyAsync(&rb.v, &s->tile_off[ntiles], 8, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaMemcpyAsync(&rb.err, &s->err, 4, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        if (rb.err) throw std::runtime_error("device error " + std::to_string(rb.err) + " in super-k-mer count");
        const uint64_t n = rb.v;
        if (n > out_cap) throw std::runtime_error("output capacity too small: need " + std::to_string(n));
        k_minimizers<1><<<(unsigned)ntiles, MZ_THREADS, mz_smem<1, MZ_TT>(), st>>>(num_runs, s->tile_start, run_soff, run_len,
                                                                 words, k, m, s->tile_count, s->tile_off,
                                                                 s->minv, s->run, s->a, &s->err);
        CDBG_CHECK_LAUNCH();
        // a tile that gave up wrote none of its cuts, and the scratch still
        // holds the previous call's entries there: stop before they are used
        CDBG_CUDA(cudaMemcpyAsync(&rb.err, &s->err, 4, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        if (rb.err) throw std::runtime_error("device error " + std::to_string(rb.err) + " in super-k-mer cuts");
        uint32_t bb = 0;
        while ((1ull << bb) < num_buckets) ++bb;
        if (n) {
            k_super_finalize<<<grid(n, 256), 256, 0, st>>>(n, s->minv, s->run, s->a, run_soff, run_len, run_color,
                                                           words, k, num_buckets, bb, out_start, out_len, out_color,
                                                           out_flags, out_bucket, s->key);
            CDBG_CHECK_LAUNCH();
        }
        uint32_t err = 0;
        CDBG_CUDA(cudaMemcpyAsync(&err, &s->err, 4, cudaMemcpyDeviceToHost, st));
        CDBG_CUDA(cudaStreamSynchronize(st));
        if (err) throw std::runtime_error("device error " + std::to_string(err) + " in super-k-mer search");
        if (n_supers) *n_supers = n;
        return 0;
    } catch (std::exception const& ex) {
        set_last_error(ex.what());  // read back with cdbg_last_error()
        return -1;
    }
}

