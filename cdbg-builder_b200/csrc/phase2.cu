// Phase 2 (bucket-process) kernels for sm_100a.
//
// Restates phase2_bucket_process/bucket_walker.hpp:166-779 on the device.
// Buckets are processed in batches (consecutive buckets whose k-mer
// occurrences fit a budget); every batch runs the same stages:
//
//  load     one thread per k-mer occurrence rolls its canonical k-mer straight
//           from the 2-bit record stream and aggregates it into its bucket's
//           open-addressing table (load_bucket, bucket_walker.hpp:166-255):
//           boundary side bits and `primary` OR-ed, the first owning record
//           plus a second-owner bit, and the first-insertion rank (the
//           occurrence index, in (record, index) order) by atomicMin.
//  nodes    distinct k-mers are numbered in first-insertion order -- the
//           iteration order of the reference's insertion-ordered map, which is
//           its seed and class order -- by marking each k-mer's first
//           occurrence in a bitmap over the batch's occurrences and scanning it.
//  resolve  a primary k-mer owned by one record has that record's color set;
//           one owned by several records gets the union of their sets
//           (bucket_walker.hpp:360-428), built once per run of k-mers with the
//           same owning records in a per-warp shared-memory bitmap.  Sets are
//           hashed (order-independent 64-bit set hash) and
//           interned in a global device dictionary with full list equality;
//           new classes get global ids in order of first appearance (bucket,
//           then insertion rank), which is the id order of the reference's
//           streaming_color_set_dict when buckets are merged in order
//           (bucket_walker.hpp:713-757, streaming_color_set_dict.hpp:148-182).
//           New classes are hybrid-encoded (hybrid_color_sets.hpp:48-95) into
//           the .color_sets bit vector.
//  walk     8-neighbour extension masks (local_ext_mask, :260-271) and the
//           clean-step links of walk_step (:317-336).  Clean links pair the
//           ports of k-mers into disjoint chains (paths and cycles); one thread
//           per chain replays the reference's sequential seed loop restricted
//           to that chain (emit_from_seed, :451-566): seeds in insertion order,
//           a shared visited set, contig-break stops and the seed shortcuts.
//           Chains never interact, so this equals the whole-bucket loop.
//  emit     fragments in seed order, serialized in the frag_unitig_writer
//           record layout (unitig_spill.hpp:491-522) with global class ids.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <vector>

#include "device_kmer.cuh"
#include "phase2.cuh"
#include "primitives.cuh"

namespace cdbg {

namespace {

constexpr uint32_t NONE32 = 0xffffffffu;
constexpr uint32_t MULTI_TAG = 0x80000000u;
constexpr uint32_t M_LEFT = 1, M_RIGHT = 2, M_PRIMARY = 4;
constexpr uint32_t M_MULTI = 8;  // table only: owned by two or more records
constexpr uint32_t SK_BEGIN = 1, SK_END = 2, SK_OWNS_FIRST = 4, SK_OWNS_LAST = 8;
constexpr uint64_t HASH_EMPTY = ~0ull;

inline unsigned grid(uint64_t n, unsigned t) { return (unsigned)ceil_div(n, t); }

template <typename T>
T read_dev(T const* p, cudaStream_t st) {
    T v;
    read_small(&v, p, sizeof(T), st);
    return v;
}

__device__ __forceinline__ uint32_t upper_bound_u64(uint64_t const* a, uint64_t n, uint64_t x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (uint32_t)lo;
}

// upper_bound(off, n1, x) - 1 (the bucket of x, `off` ascending) for the
// active lanes of a warp whose x ascend with the lane (consecutive records or
// occurrences, so nearly always one bucket): the first active lane searches,
// the others take its bucket when x lies in its range and search otherwise.
// Every lane of the warp calls it.
__device__ __forceinline__ uint32_t warp_bucket_of(uint64_t const* off, uint64_t n1, uint64_t x, bool active) {
    const uint32_t am = __ballot_sync(0xffffffffu, active);
    if (!am) return 0;
    const int leader = __ffs(am) - 1;
    const uint64_t xl = __shfl_sync(0xffffffffu, x, leader);
    uint32_t b = 0;
    if ((int)(threadIdx.x & 31) == leader) b = upper_bound_u64(off, n1, xl) - 1;
    b = __shfl_sync(0xffffffffu, b, leader);
    if (active && !(off[b] <= x && x < off[b + 1])) b = upper_bound_u64(off, n1, x) - 1;
    return b;
}

// ------------------------------------------------------------------ set hash
// Order-independent hash of a color set: the sum, over the 32-color words
// that hold at least one color, of a mix of (word index, word bits), then
// mixed with the set size.  A list and a bitmap of the same set hash alike;
// one mix per nonzero word instead of one per color.
__host__ __device__ __forceinline__ uint64_t word_mix(uint32_t w, uint32_t bits) {
    return mix64((((uint64_t)w << 32) | bits) * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL);
}
// Sum of word_mix over an ascending color list.
__host__ __device__ __forceinline__ uint64_t list_word_sum(uint32_t const* c, uint64_t n) {
    uint64_t acc = 0;
    uint32_t cw = 0xffffffffu, bits = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t v = c[i], w = v >> 5;
        if (w != cw) {
            if (bits) acc += word_mix(cw, bits);
            cw = w;
            bits = 0;
        }
        bits |= 1u << (v & 31);
    }
    if (bits) acc += word_mix(cw, bits);
    return acc;
}
__host__ __device__ __forceinline__ uint64_t set_hash_final(uint64_t acc, uint64_t n) {
    uint64_t h = mix64(acc ^ (n * 0xD6E8FEB86659FD93ULL));
    return h == HASH_EMPTY ? HASH_EMPTY - 1 : h;
}

// ------------------------------------------------------------------ tables
__device__ __forceinline__ u128 key_cas(u128* a, u128 cmp, u128 val) {
    uint64_t olo, ohi;
    const uint64_t clo = (uint64_t)cmp, chi = (uint64_t)(cmp >> 64);
    const uint64_t vlo = (uint64_t)val, vhi = (uint64_t)(val >> 64);
    asm volatile(
        "{\n\t.reg .b128 d, c, v;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 v, {%4, %5};\n\t"
        "atom.global.cas.b128 d, [%6], c, v;\n\t"
        "mov.b128 {%0, %1}, d;\n\t}"
        : "=l"(olo), "=l"(ohi)
        : "l"(clo), "l"(chi), "l"(vlo), "l"(vhi), "l"(a)
        : "memory");
    return ((u128)ohi << 64) | (u128)olo;
}

// One table slot: everything the load stage aggregates for a k-mer in 16
// bytes (32 for 128-bit k-mers), two slots per 32-byte sector.
//   rank  first insertion: the batch's lowest occurrence index of the k-mer
//         (occurrences are in (record, index) order); after numbering, the
//         k-mer's node index
//   om    bits 0-3: side bits, primary, M_MULTI; bits 4-31: the first owning
//         record (relative to the batch) + 1, 0 when none
template <typename K>
struct slot_t;
template <>
struct alignas(16) slot_t<uint64_t> {
    uint64_t key;
    uint32_t rank;
    uint32_t om;
};
template <>
struct alignas(16) slot_t<u128> {
    u128 key;
    uint32_t rank;
    uint32_t om;
    uint64_t pad;
};
static_assert(sizeof(slot_t<uint64_t>) == 16, "slot layout");
static_assert(sizeof(slot_t<u128>) == 32, "slot layout");
constexpr uint64_t MAX_BATCH_RECORDS = (1ull << 28) - 2;  // owner field of `om`

// First slot of key x in a table of `cap` slots (cap < 2^32): the key folded
// to 64 bits, an odd-constant multiply, and its top 32 bits scaled to the
// capacity.  Table positions decide no output (nodes are numbered by first
// occurrence, not by slot), only probe lengths.
__device__ __forceinline__ uint32_t slot_of(uint64_t x, uint32_t cap) {
    const uint64_t h = (x ^ (x >> 31)) * 0x9e3779b97f4a7c15ULL;
    return (uint32_t)(((h >> 32) * (uint64_t)cap) >> 32);
}
__device__ __forceinline__ uint32_t slot_of(u128 x, uint32_t cap) {
    const uint64_t f = (uint64_t)x ^ ((uint64_t)(x >> 64) * 0xc2b2ae3d27d4eb4fULL);
    return slot_of(f, cap);
}

// A 64-bit-key slot's key and (rank | om << 32) in one 16-byte load that
// bypasses L1.
__device__ __forceinline__ void slot_load(slot_t<uint64_t> const* e, uint64_t& key, uint64_t& ro) {
    asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];" : "=l"(key), "=l"(ro) : "l"(e) : "memory");
}

// Insert-or-find; returns the slot (absolute) or NONE64 when the region is
// full.  `ro` receives the slot's (rank | om << 32) as read while probing: a
// value the slot held, so possibly older than the current one (rank only
// falls and om only gains bits, which the caller's updates rely on).
// `slots` holds the slots from absolute index off0 on (the tables of the
// bucket group being processed); returned indices are absolute.
template <typename K>
__device__ __forceinline__ uint64_t table_upsert(slot_t<K>* slots, uint64_t off0, uint64_t off, uint64_t cap, K x,
                                                 uint64_t& ro) {
    const K EMPTY = kmer_ops<K>::empty();
    const uint32_t cap32 = (uint32_t)cap;
    uint32_t s = slot_of(x, cap32);
    for (uint32_t i = 0; i < cap32; ++i) {
        slot_t<K>* e = &slots[off + s - off0];
        if constexpr (sizeof(K) == 8) {
            uint64_t cur, v;
            slot_load(e, cur, v);
            if (cur == x) {
                ro = v;
                return off + s;
            }
            if (cur == EMPTY) {
                const K old = (K)atomicCAS((unsigned long long*)&e->key, (unsigned long long)EMPTY,
                                           (unsigned long long)x);
                if (old == EMPTY || old == x) {
                    ro = v;
                    return off + s;
                }
            }
        } else {
            const K old = key_cas(&e->key, EMPTY, x);  // atomic 128-bit read-or-claim
            if (old == EMPTY || old == x) {
                ro = *(volatile uint64_t const*)&e->rank;
                return off + s;
            }
        }
        s = s + 1 == cap32 ? 0u : s + 1;
    }
    return ~0ull;
}

// 64-bit-key tables: insert-or-find like table_upsert, but an empty slot is
// claimed together with the payload a new k-mer gets -- its rank and om --
// in one 128-bit compare-and-swap of the whole slot (key, rank, om), so the
// occurrence that creates a k-mer needs no further atomics.  `claimed` tells
// whether this call wrote the payload; otherwise `ro` is the slot's (rank |
// om << 32) as read (the caller's updates as in table_upsert).
__device__ __forceinline__ uint64_t table_claim(slot_t<uint64_t>* slots, uint64_t off0, uint64_t off, uint64_t cap,
                                                uint64_t x, uint64_t payload, uint64_t& ro, bool& claimed) {
    const uint64_t EMPTY = kmer_ops<uint64_t>::empty();
    const uint32_t cap32 = (uint32_t)cap;
    uint32_t s = slot_of(x, cap32);
    claimed = false;
    for (uint32_t i = 0; i < cap32; ++i) {
        slot_t<uint64_t>* e = &slots[off + s - off0];
        uint64_t cur, v;
        slot_load(e, cur, v);
        if (cur == x) {
            ro = v;
            return off + s;
        }
        if (cur == EMPTY) {
            const u128 old = key_cas(reinterpret_cast<u128*>(e), ((u128)v << 64) | (u128)EMPTY,
                                     ((u128)payload << 64) | (u128)x);
            if ((uint64_t)old == EMPTY && (uint64_t)(old >> 64) == v) {
                claimed = true;
                return off + s;
            }
            if ((uint64_t)old == x) {
                ro = (uint64_t)(old >> 64);
                return off + s;
            }
        }
        s = s + 1 == cap32 ? 0u : s + 1;
    }
    return ~0ull;
}

struct rec_view {
    uint64_t const* start;
    uint32_t const* len;
    uint32_t const* flags;
    uint64_t const* col_off;
    uint32_t const* colors;
    uint32_t const* bucket;   // per record
    uint64_t const* occ;      // n + 1 exclusive prefix of k-mers per record
    uint64_t const* words;
};

// The k-mer tables of buckets b0, b0 + 1, ...: bucket b0 + i's table is
// the tab_cap[i] slots from absolute slot tab_off[i]; `slots` holds the slots
// from absolute index off0 on (one bucket group's tables at a time).
template <typename K>
struct tables {
    slot_t<K>* slots;
    uint64_t const* tab_off;
    uint64_t const* tab_cap;
    uint32_t b0;
    uint64_t off0;
};

// Occurrence o of the batch -> (record, index, canonical k-mer, contrib, owned).
template <typename K>
struct occ_info {
    uint32_t r;
    uint32_t idx;
    K can;
    uint32_t contrib;
    bool owned;
};

// Record holding occurrence o of the current block.  Every record has at least
// one k-mer in practice, so the block's OCC_BLOCK occurrences fall within
// OCC_BLOCK + 1 records starting at the record of its first occurrence: one
// global binary search per block, then a search in shared memory.  Empty
// records (len < k) can push an occurrence past the window; it then falls
// back to the global search.
constexpr int OCC_BLOCK = 256;
struct occ_window {
    uint64_t occ[OCC_BLOCK + 2];
    uint64_t r0;
};
// blk_rec[b] = the record holding occurrence O0 + b * OCC_BLOCK, the first
// occurrence of block b of the occurrence kernels (thread per record; a
// record spans at most a few block starts).
__global__ void k_block_records(uint64_t const* __restrict__ occ, uint64_t R0, uint64_t nrec, uint64_t O0,
                                uint64_t nblocks, uint32_t* __restrict__ blk_rec) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrec) return;
    const uint64_t a = occ[R0 + i] - O0, e = occ[R0 + i + 1] - O0;
    for (uint64_t b = (a + OCC_BLOCK - 1) / OCC_BLOCK; b * OCC_BLOCK < e && b < nblocks; ++b)
        blk_rec[b] = (uint32_t)(R0 + i);
}

__device__ __forceinline__ void load_occ_window(occ_window& w, uint64_t const* occ, uint64_t R0, uint64_t nrec,
                                                uint32_t const* __restrict__ blk_rec, uint64_t blk) {
    if (threadIdx.x == 0) w.r0 = blk_rec[blk];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < OCC_BLOCK + 2; i += blockDim.x) {
        const uint64_t r = w.r0 + i;
        w.occ[i] = (r <= R0 + nrec) ? occ[r] : ~0ull;
    }
    __syncthreads();
}
__device__ __forceinline__ uint64_t window_record(occ_window const& w, uint64_t const* occ, uint64_t R0,
                                                  uint64_t nrec, uint64_t o) {
    if (o < w.occ[OCC_BLOCK + 1]) {
        uint32_t lo = 0, hi = OCC_BLOCK + 2;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (w.occ[mid] <= o)
                lo = mid + 1;
            else
                hi = mid;
        }
        return w.r0 + lo - 1;
    }
    return R0 + upper_bound_u64(occ + R0, nrec + 1, o) - 1;
}

template <typename K>
__device__ __forceinline__ occ_info<K> decode_occ_r(rec_view const& R, uint64_t r, uint64_t o, uint32_t k) {
    occ_info<K> oi;
    oi.r = (uint32_t)r;
    oi.idx = (uint32_t)(o - R.occ[r]);
    const uint32_t nk = R.len[r] - k + 1;
    const uint32_t f = R.flags[r];
    K fwd, rc;
    kmer_ops<K>::load(R.words, R.start[r] + oi.idx, k, fwd, rc);
    const bool isf = fwd <= rc;
    oi.can = isf ? fwd : rc;
    uint32_t contrib = 0;
    if (!(f & SK_BEGIN) && oi.idx == 0) contrib |= isf ? M_LEFT : M_RIGHT;
    if (!(f & SK_END) && oi.idx == nk - 1) contrib |= isf ? M_RIGHT : M_LEFT;
    oi.contrib = contrib;
    oi.owned = !((oi.idx == 0 && !(f & SK_OWNS_FIRST)) || (oi.idx == nk - 1 && !(f & SK_OWNS_LAST)));
    return oi;
}

// ------------------------------------------------------------------ kernels
__global__ void k_rec_prep(uint64_t n, uint32_t const* __restrict__ len, uint32_t k,
                           uint64_t const* __restrict__ bstart, uint32_t B,
                           uint64_t* __restrict__ nk, uint32_t* __restrict__ rbucket,
                           uint64_t const* __restrict__ col_off, uint32_t const* __restrict__ colors,
                           uint64_t* __restrict__ rhash) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t b = warp_bucket_of(bstart, (uint64_t)B + 1, r, r < n);
    if (r >= n) return;
    const uint32_t l = len[r];
    nk[r] = l >= k ? (uint64_t)(l - k + 1) : 0;
    rbucket[r] = b;
    const uint64_t c0 = col_off[r], c1 = col_off[r + 1];
    rhash[r] = set_hash_final(list_word_sum(colors + c0, c1 - c0), c1 - c0);
}

__global__ void k_gather_u64(uint64_t n, uint64_t const* __restrict__ src,
                             uint64_t const* __restrict__ idx, uint64_t* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[idx[i]];
}

template <typename K>
__global__ void k_init_tables(uint64_t T, slot_t<K>* slots) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    slot_t<K> e;
    e.key = kmer_ops<K>::empty();
    e.rank = NONE32;
    e.om = 0;
    if constexpr (sizeof(K) == 16) e.pad = 0;
    slots[i] = e;
}

// Occurrences t0 .. t0 + nocc - 1 of the batch (one bucket group's).
template <typename K>
__global__ void __launch_bounds__(256) k_insert(rec_view R, tables<K> T, uint64_t R0, uint64_t nrec,
                                                uint64_t O0, uint64_t t0, uint64_t nocc, uint32_t k,
                                                uint32_t const* __restrict__ blk_rec,
                                                uint32_t* __restrict__ occ_slot, uint32_t* err) {
    __shared__ occ_window win;
    // the window of the occurrence block holding this block's first occurrence
    load_occ_window(win, R.occ, R0, nrec, blk_rec, (t0 + (uint64_t)blockIdx.x * blockDim.x) / OCC_BLOCK);
    const uint64_t t = t0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= t0 + nocc) return;
    const uint64_t rec = window_record(win, R.occ, R0, nrec, O0 + t);
    const occ_info<K> oi = decode_occ_r<K>(R, rec, O0 + t, k);
    const uint32_t tb = R.bucket[oi.r] - T.b0;
    const uint32_t mo = oi.contrib | (oi.owned ? M_PRIMARY : 0u);
    const uint32_t own = (uint32_t)(oi.r - R0 + 1) << 4;
    uint64_t ro = 0;
    bool claimed = false;
    uint64_t s;
    if constexpr (sizeof(K) == 8) {
        // a new k-mer's slot: rank t, and om as the updates below would leave it
        const uint32_t om0 = oi.owned ? (own | mo) : mo;
        s = table_claim(T.slots, T.off0, T.tab_off[tb], T.tab_cap[tb], oi.can,
                        (uint64_t)(uint32_t)t | ((uint64_t)om0 << 32), ro, claimed);
    } else {
        s = table_upsert<K>(T.slots, T.off0, T.tab_off[tb], T.tab_cap[tb], oi.can, ro);
    }
    if (s == ~0ull) {
        set_error(err, ERR_TABLE_FULL);
        occ_slot[t] = NONE32;
        return;
    }
    // slot of this occurrence, bit 31 = owned (read by k_multi_pairs)
    occ_slot[t] = (uint32_t)s | (oi.owned ? 0x80000000u : 0u);
    if (claimed) return;
    // rank and om as read while probing (never newer than the slot): the
    // reduction and the updates below stay correct, and a k-mer whose slot
    // already holds everything this occurrence adds costs no further access
    slot_t<K>& e = T.slots[s - T.off0];
    if ((uint32_t)t < (uint32_t)ro) atomicMin(&e.rank, (uint32_t)t);
    uint32_t old = (uint32_t)(ro >> 32);
    if (!oi.owned) {
        if (mo && (old & mo) != mo) atomicOr(&e.om, mo);
        return;
    }
    // owner: the first owning record, M_MULTI once a second one appears.
    // `om` only gains bits, so the loop ends after a few changes by others.
    for (int it = 0;; ++it) {
        const uint32_t cur = old & ~0xfu;
        const uint32_t want = (cur == own || (old & M_MULTI)) ? (old | mo)
                              : (cur == 0)                   ? (old | own | mo)
                                                             : (old | M_MULTI | mo);
        if (want == old) break;
        const uint32_t prev = atomicCAS(&e.om, old, want);
        if (prev == old) break;
        old = prev;
        if (it == 64) {
            set_error(err, ERR_CAPACITY);
            break;
        }
    }
}

// Bit q of `bits` <- first occurrence of each distinct k-mer.
template <typename K>
__global__ void k_firstbits(uint64_t T, slot_t<K> const* __restrict__ slots, uint32_t* __restrict__ bits) {
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= T || slots[s].key == kmer_ops<K>::empty()) return;
    const uint32_t q = slots[s].rank;
    atomicOr(&bits[q >> 5], 1u << (q & 31));
}


// Number the distinct k-mers of one bucket group in first-insertion order,
// scanning its occurrences t0 .. t0 + nocc - 1: occurrence t is the first of
// its k-mer iff bit t of `bits` is set, and its node index is *nbase plus the
// number of first occurrences before it in the group.  Tiles of MN_ROUNDS x
// 256 occurrences take indices in launch order and find their offset by
// decoupled look-back; the last tile stores *nbase + the group's count in
// *nnext (the next group's base).  The slot's rank field becomes the node
// index, and the node arrays are written in node order; the bucket is the
// slot's table (tab_off ascends over the group's buckets).
constexpr int MN_ROUNDS = 8;
template <typename K>
__global__ void __launch_bounds__(256) k_make_nodes(uint64_t t0, uint64_t nocc, uint32_t const* __restrict__ occ_slot,
                                                    uint32_t const* __restrict__ bits, tables<K> TB, uint32_t nb,
                                                    uint64_t R0, unsigned long long const* nbase,
                                                    unsigned long long* nnext, uint32_t* tile_counter,
                                                    unsigned long long* status, K* __restrict__ n_key,
                                                    uint8_t* __restrict__ n_meta, uint32_t* __restrict__ n_rec,
                                                    uint32_t* __restrict__ n_bucket, uint32_t* err) {
    constexpr int NW = 256 / 32;
    static_assert(MN_ROUNDS * NW == 64, "warp 0 scans two counts per lane");
    __shared__ uint64_t s_tile;
    __shared__ uint32_t wcnt[MN_ROUNDS * NW];
    __shared__ unsigned long long s_base;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t ntiles = (nocc + MN_ROUNDS * 256 - 1) / (MN_ROUNDS * 256);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t rank[MN_ROUNDS], first = 0;
#pragma unroll
    for (int rr = 0; rr < MN_ROUNDS; ++rr) {
        const uint64_t l = (tile * MN_ROUNDS + rr) * 256 + threadIdx.x;
        const uint64_t t = t0 + l;
        const bool f = l < nocc && ((bits[t >> 5] >> (t & 31)) & 1u);
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        rank[rr] = __popc(bal & lanemask_lt());
        if (f) first |= 1u << rr;
        if (lane == 0) wcnt[rr * NW + warp] = __popc(bal);
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t c0 = wcnt[2 * lane], c1 = wcnt[2 * lane + 1];
        uint32_t x = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
        const uint32_t ex = x - c0 - c1;
        wcnt[2 * lane] = ex;
        wcnt[2 * lane + 1] = ex + c0;
        uint64_t excl = 0;
        const bool ok = prim::lookback_exclusive(status, tile, tot, excl);
        if (lane == 0) {
            if (!ok) set_error(err, ERR_CHAIN_LIMIT);
            s_base = *nbase + excl;
            if (tile == ntiles - 1) *nnext = *nbase + excl + tot;
        }
    }
    __syncthreads();
    const unsigned long long base = s_base;
    // every round's slot loads go out before any store, so a thread keeps
    // its MN_ROUNDS random slot reads in flight at once
    uint32_t sl[MN_ROUNDS];
#pragma unroll
    for (int rr = 0; rr < MN_ROUNDS; ++rr) {
        const uint64_t t = t0 + (tile * MN_ROUNDS + rr) * 256 + threadIdx.x;
        sl[rr] = ((first >> rr) & 1u) ? __ldg(occ_slot + t) & 0x7fffffffu : 0u;
    }
    K key[MN_ROUNDS];
    uint32_t om[MN_ROUNDS];
#pragma unroll
    for (int rr = 0; rr < MN_ROUNDS; ++rr) {
        if ((first >> rr) & 1u) {
            slot_t<K> const* e = TB.slots + (sl[rr] - TB.off0);
            key[rr] = e->key;
            om[rr] = e->om;
        }
    }
#pragma unroll
    for (int rr = 0; rr < MN_ROUNDS; ++rr) {
        const bool f = (first >> rr) & 1u;
        const uint32_t tb = warp_bucket_of(TB.tab_off, nb + 1, sl[rr], f);
        if (!f) continue;
        const uint64_t n = base + wcnt[rr * NW + warp] + rank[rr];
        TB.slots[sl[rr] - TB.off0].rank = (uint32_t)n;
        n_key[n] = key[rr];
        n_meta[n] = (uint8_t)(om[rr] & 7u);
        uint32_t rec = NONE32;
        if (om[rr] & M_PRIMARY) rec = (om[rr] & M_MULTI) ? MULTI_TAG : (uint32_t)(R0 + (om[rr] >> 4) - 1);
        n_rec[n] = rec;
        n_bucket[n] = TB.b0 + tb;
    }
}

// Occurrences t0 .. t0 + nocc - 1: the slot index becomes the k-mer's node
// index (bit 31, owned, kept), so later stages need no table.
template <typename K>
__global__ void k_occ_nodes(uint64_t t0, uint64_t nocc, uint32_t* __restrict__ occ_slot,
                            slot_t<K> const* __restrict__ slots, uint64_t off0) {
    const uint64_t t = t0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= t0 + nocc) return;
    const uint32_t v = occ_slot[t];
    if (v == NONE32) return;
    occ_slot[t] = slots[(v & 0x7fffffffu) - off0].rank | (v & 0x80000000u);
}

// Block-wide reservation of `want` consecutive entries of *cnt per thread,
// one atomic per block (a counter shared by millions of warps serializes
// their atomics).  Every thread of the block must call it.
template <int THREADS>
__device__ __forceinline__ unsigned long long block_reserve(uint32_t want, unsigned long long* cnt) {
    __shared__ unsigned long long s_warp[THREADS / 32];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long incl = want;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int w = 0; w < THREADS / 32; ++w) {
            const unsigned long long v = s_warp[w];
            s_warp[w] = run;
            run += v;
        }
        s_base = run ? atomicAdd(cnt, run) : 0ull;
    }
    __syncthreads();
    const unsigned long long r = s_base + s_warp[warp] + incl - want;
    __syncthreads();  // the shared words may be reused by the next call
    return r;
}

// (node, record) of the owned occurrences of multi-record k-mers, from the
// slot each occurrence recorded at insert time, written in occurrence order
// (records ascend within a node, so a stable sort by node alone orders the
// pairs by (node, record)).  A block handles MP_ROUNDS consecutive
// occurrence blocks of OCC_BLOCK (one per round); blocks take tile indices in
// launch order and find their output offset by decoupled look-back; the grid
// is exactly one block per tile.
constexpr int MP_ROUNDS = 8;
__global__ void __launch_bounds__(OCC_BLOCK)
    k_multi_pairs(uint64_t const* __restrict__ occ, uint64_t R0, uint64_t nrec, uint64_t O0, uint64_t nocc,
                  uint32_t const* __restrict__ blk_rec,
                  uint32_t const* __restrict__ occ_slot, uint32_t const* __restrict__ slot_rank, uint32_t rank_stride,
                  uint32_t const* __restrict__ n_rec, uint32_t* __restrict__ tile_counter,
                  unsigned long long* __restrict__ status, unsigned long long* __restrict__ cnt,
                  uint32_t* __restrict__ pnode, uint32_t* __restrict__ prec, uint64_t cap, uint32_t* err) {
    constexpr int NW = OCC_BLOCK / 32;
    static_assert(MP_ROUNDS * NW == 64, "warp 0 scans two counts per lane");
    __shared__ uint64_t s_tile;
    __shared__ uint32_t wcnt[MP_ROUNDS * NW];
    __shared__ unsigned long long s_base;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t nblk = (nocc + OCC_BLOCK - 1) / OCC_BLOCK;
    uint32_t node[MP_ROUNDS], rec[MP_ROUNDS], rank[MP_ROUNDS], emit = 0;
#pragma unroll
    for (int rr = 0; rr < MP_ROUNDS; ++rr) {
        const uint64_t b = tile * MP_ROUNDS + rr;  // occurrence block
        const uint64_t t = b * OCC_BLOCK + threadIdx.x;
        bool e = false;
        node[rr] = 0;
        rec[rr] = 0;
        if (t < nocc) {
            const uint32_t v = occ_slot[t];
            if (v != NONE32 && (v & 0x80000000u)) {
                uint32_t n;
                bool multi;
                if (slot_rank) {
                    // the slot's node index and owner bits in one load: a
                    // multi-record k-mer has both M_PRIMARY and M_MULTI (the
                    // MULTI_TAG k_make_nodes writes to n_rec)
                    const uint2 ro = __ldg(reinterpret_cast<uint2 const*>(
                        slot_rank + (uint64_t)(v & 0x7fffffffu) * rank_stride));
                    n = ro.x;
                    multi = (ro.y & (M_PRIMARY | M_MULTI)) == (M_PRIMARY | M_MULTI);
                } else {
                    n = v & 0x7fffffffu;
                    multi = n_rec[n] == MULTI_TAG;
                }
                if (multi) {
                    // the record lies between this occurrence block's first record
                    // and the next one's (a few dozen records): search only there
                    const uint64_t rlo = blk_rec[b];
                    const uint64_t rhi = (b + 1 < nblk) ? blk_rec[b + 1] : R0 + nrec - 1;
                    node[rr] = n;
                    rec[rr] = (uint32_t)(rlo + upper_bound_u64(occ + rlo, rhi - rlo + 1, O0 + t) - 1);
                    e = true;
                }
            }
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, e);
        rank[rr] = __popc(bal & lanemask_lt());
        if (e) emit |= 1u << rr;
        if (lane == 0) wcnt[rr * NW + warp] = __popc(bal);
    }
    __syncthreads();
    if (warp == 0) {
        // exclusive prefix of the (round, warp) counts in position order
        const uint32_t c0 = wcnt[2 * lane], c1 = wcnt[2 * lane + 1];
        uint32_t x = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
        const uint32_t ex = x - c0 - c1;
        wcnt[2 * lane] = ex;
        wcnt[2 * lane + 1] = ex + c0;
        uint64_t excl = 0;
        const bool ok = prim::lookback_exclusive(status, tile, tot, excl);
        if (lane == 0) {
            if (!ok) set_error(err, ERR_CHAIN_LIMIT);
            if (tot) atomicAdd(cnt, (unsigned long long)tot);
            s_base = excl;
        }
    }
    __syncthreads();
    const unsigned long long base = s_base;
#pragma unroll
    for (int rr = 0; rr < MP_ROUNDS; ++rr) {
        if (!((emit >> rr) & 1u)) continue;
        const unsigned long long at = base + wcnt[rr * NW + warp] + rank[rr];
        if (at < cap) {
            pnode[at] = node[rr];
            prec[at] = rec[rr];
        }
    }
}

// First of each run of equal (node, record) pairs (a record may own a k-mer
// at two positions).
__global__ void k_unique_pairs(uint64_t n, uint32_t const* __restrict__ pn, uint32_t const* __restrict__ pr,
                               uint32_t* __restrict__ keep) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keep[i] = (i == 0 || pn[i] != pn[i - 1] || pr[i] != pr[i - 1]) ? 1u : 0u;
}

// Kept pairs as (node << 32 | record).
__global__ void k_compact_pairs(uint64_t n, uint32_t const* __restrict__ pn, uint32_t const* __restrict__ pr,
                                uint32_t const* __restrict__ keep, uint64_t const* __restrict__ pos,
                                uint64_t* __restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && keep[i]) out[pos[i]] = ((uint64_t)pn[i] << 32) | pr[i];
}

__global__ void k_node_heads(uint64_t n, uint64_t const* __restrict__ a, uint32_t* __restrict__ head) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || (a[i] >> 32) != (a[i - 1] >> 32)) ? 1u : 0u;
}

// Multi-record nodes: m-th head -> node id, record range [moff[m], moff[m+1]).
__global__ void k_multi_index(uint64_t n, uint64_t const* __restrict__ a, uint32_t const* __restrict__ head,
                              uint64_t const* __restrict__ hpos, uint32_t* __restrict__ mnode,
                              uint64_t* __restrict__ moff, uint32_t* __restrict__ n_rec) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    const uint64_t m = hpos[i];
    const uint32_t node = (uint32_t)(a[i] >> 32);
    mnode[m] = node;
    moff[m] = i;
    n_rec[node] = MULTI_TAG | (uint32_t)m;
}

// Multi-record nodes in node order whose owning-record list equals the
// previous one's (the k-mers of a stretch shared by the same records) share
// one union: ghead[m] = 1 starts a new group.
__global__ void k_multi_same(uint64_t M, uint64_t const* __restrict__ moff, uint64_t const* __restrict__ upairs,
                             uint32_t* __restrict__ ghead) {
    uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    bool same = false;
    if (m > 0) {
        const uint64_t a0 = moff[m - 1], a1 = moff[m], b1 = moff[m + 1];
        if (a1 - a0 == b1 - a1) {
            same = true;
            for (uint64_t i = 0; i < a1 - a0; ++i)
                if ((uint32_t)upairs[a0 + i] != (uint32_t)upairs[a1 + i]) {
                    same = false;
                    break;
                }
        }
    }
    ghead[m] = same ? 0u : 1u;
}

// Group g (of its head node m): node, record range; every multi node's group.
__global__ void k_multi_groups(uint64_t M, uint32_t const* __restrict__ ghead, uint64_t const* __restrict__ gpos,
                               uint32_t const* __restrict__ mnode, uint64_t const* __restrict__ moff,
                               uint32_t* __restrict__ gnode, uint64_t* __restrict__ gbeg, uint64_t* __restrict__ gend,
                               uint32_t* __restrict__ mgrp) {
    uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const uint64_t g = gpos[m] + ghead[m] - 1;
    mgrp[m] = (uint32_t)g;
    if (ghead[m]) {
        gnode[g] = mnode[m];
        gbeg[g] = moff[m];
        gend[g] = moff[m + 1];
    }
}

// Warp-level helpers over a per-warp shared-memory bitmap of C bits.
__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ uint32_t warp_excl_scan32(uint32_t v, uint32_t& total) {
    const int lane = threadIdx.x & 31;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}
__device__ __forceinline__ uint64_t warp_excl_scan64(uint64_t v, uint64_t& total) {
    const int lane = threadIdx.x & 31;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// OR the ascending list [c0, c1) of `list` into the shared bitmap `bm` of
// `nw` words (all 32 lanes call it).  A dense list (at least one element per
// 4 bit positions: 8 or more lanes per word) has the lanes holding the same
// word (consecutive lanes) combine their bits first, the first of them alone
// touching shared memory; a sparser one ORs lane by lane.  An unsorted list
// is ORed correctly either way.
__device__ __forceinline__ void warp_or_list(uint32_t* bm, uint32_t const* __restrict__ list, uint64_t c0,
                                             uint64_t c1, uint32_t nw, int lane) {
    if ((c1 - c0) * 4 < (uint64_t)nw * 32) {
        for (uint64_t c = c0 + lane; c < c1; c += 32) {
            const uint32_t v = list[c];
            atomicOr(&bm[v >> 5], 1u << (v & 31));
        }
        return;
    }
    for (uint64_t base = c0; base < c1; base += 32) {
        const bool in = base + lane < c1;
        const uint32_t v = in ? list[base + lane] : NONE32;
        const uint32_t w = v >> 5;
        uint32_t b = in ? 1u << (v & 31) : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ob = __shfl_down_sync(0xffffffffu, b, o);
            const uint32_t ow = __shfl_down_sync(0xffffffffu, w, o);
            if (lane + o < 32 && ow == w) b |= ob;
        }
        const uint32_t pw = __shfl_up_sync(0xffffffffu, w, 1);
        if (in && (lane == 0 || pw != w)) atomicOr(&bm[w], b);
    }
}

// Union of the color lists of a multi-record node.  Pass 0: size and hash;
// pass 1: write the ascending list at pool[poff[m]].
template <bool WRITE>
__global__ void k_union(uint64_t M, uint64_t const* __restrict__ mbeg, uint64_t const* __restrict__ mend,
                        uint64_t const* __restrict__ upairs,
                        uint64_t const* __restrict__ col_off, uint32_t const* __restrict__ colors,
                        uint32_t C, uint32_t* __restrict__ msize, uint64_t* __restrict__ mhash,
                        uint64_t const* __restrict__ poff, uint32_t* __restrict__ pool) {
    extern __shared__ uint32_t smem_bm[];
    const uint32_t nw = (C + 31) / 32;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* bm = smem_bm + (size_t)wib * nw;
    const uint64_t m = (uint64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (m >= M) return;
    for (uint32_t w = lane; w < nw; w += 32) bm[w] = 0;
    __syncwarp();
    for (uint64_t p = mbeg[m]; p < mend[m]; ++p) {
        const uint32_t r = (uint32_t)(upairs[p] & 0xffffffffu);
        warp_or_list(bm, colors, col_off[r], col_off[r + 1], nw, lane);
    }
    __syncwarp();
    const uint32_t per = (nw + 31) / 32;
    const uint32_t w0 = lane * per, w1 = min(w0 + per, nw);
    uint32_t cnt = 0;
    uint64_t acc = 0;
    for (uint32_t w = w0; w < w1; ++w) {
        uint32_t x = bm[w];
        cnt += __popc(x);
        if (!WRITE && x) acc += word_mix(w, x);
    }
    uint32_t total;
    const uint32_t ex = warp_excl_scan32(cnt, total);
    if (!WRITE) {
        acc = warp_sum64(acc);
        if (lane == 0) {
            msize[m] = total;
            mhash[m] = set_hash_final(acc, total);
        }
    } else {
        uint32_t* out = pool + poff[m] + ex;
        for (uint32_t w = w0; w < w1; ++w) {
            uint32_t x = bm[w];
            while (x) {
                const uint32_t b = __ffs(x) - 1;
                x &= x - 1;
                *out++ = w * 32 + b;
            }
        }
    }
}

// ---- multi-record unions as bitmaps -----------------------------------------
// Records with at least `heavy` colors get a bitmap.
__global__ void k_heavy_flags(uint64_t nu, uint64_t const* __restrict__ upairs, uint64_t const* __restrict__ col_off,
                              uint32_t R0, uint32_t heavy, uint32_t* __restrict__ flag) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nu) return;
    const uint32_t r = (uint32_t)(upairs[i] & 0xffffffffu);
    if (col_off[r + 1] - col_off[r] >= heavy) flag[r - R0] = 1u;
}

// Heavy records' colors as bitmaps in rbits[hpos[r - R0] * nw].
__global__ void k_heavy_bitmaps(uint64_t nrec, uint32_t const* __restrict__ flag, uint64_t const* __restrict__ hpos,
                                uint32_t R0, uint64_t const* __restrict__ col_off, uint32_t const* __restrict__ colors,
                                uint32_t nw, uint32_t* __restrict__ rbits) {
    extern __shared__ uint32_t smem_bm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* bm = smem_bm + (size_t)wib * nw;
    // 32 records per warp: the lanes read the flags at once (few records are
    // heavy), then the warp builds each heavy record's bitmap
    const uint64_t i0 = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + wib) * 32;
    if (i0 >= nrec) return;
    uint32_t fm = __ballot_sync(0xffffffffu, i0 + lane < nrec && flag[i0 + lane]);
    while (fm) {
        const uint64_t i = i0 + (uint32_t)(__ffs(fm) - 1);
        fm &= fm - 1;
        for (uint32_t w = lane; w < nw; w += 32) bm[w] = 0;
        __syncwarp();
        warp_or_list(bm, colors, col_off[R0 + i], col_off[R0 + i + 1], nw, lane);
        __syncwarp();
        uint32_t* out = rbits + hpos[i] * (uint64_t)nw;
        for (uint32_t w = lane; w < nw; w += 32) out[w] = bm[w];
        __syncwarp();
    }
}

// Warp per multi-record node: OR of its records' color sets (bitmap words for
// heavy records, per-color bits for the rest) -> mbits, size, set hash.
// The records' metadata is fetched 32 at a time, one record per lane; heavy
// records' bitmap words are ORed into registers (lane owns words lane + 32u,
// u < WPL), four records' lines in flight at a time; the rest have their
// colors spread over the lanes and set bits in the warp's shared bitmap.
template <int WPL>
__global__ void __launch_bounds__(256) k_union_bm(
    uint64_t M, uint64_t const* __restrict__ mbeg, uint64_t const* __restrict__ mend,
    uint64_t const* __restrict__ upairs, uint64_t const* __restrict__ col_off, uint32_t const* __restrict__ colors,
    uint32_t R0, uint32_t const* __restrict__ hflag, uint64_t const* __restrict__ hpos,
    uint32_t const* __restrict__ rbits, uint32_t nw, uint32_t* __restrict__ mbits, uint32_t* __restrict__ msize,
    uint64_t* __restrict__ mhash) {
    extern __shared__ uint32_t smem_bm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* bm = smem_bm + (size_t)wib * nw;
    const uint64_t m = (uint64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (m >= M) return;
    for (uint32_t w = lane; w < nw; w += 32) bm[w] = 0;
    __syncwarp();
    uint32_t acc[WPL];
#pragma unroll
    for (int u = 0; u < WPL; ++u) acc[u] = 0;
    const uint64_t pend = mend[m];
    for (uint64_t p0 = mbeg[m]; p0 < pend; p0 += 32) {
        const uint64_t p = p0 + lane;
        bool heavy = false, light = false;
        uint64_t src = 0, c0 = 0, c1 = 0;
        if (p < pend) {
            const uint32_t r = (uint32_t)(upairs[p] & 0xffffffffu);
            heavy = hflag[r - R0] != 0;
            light = !heavy;
            if (heavy) {
                src = hpos[r - R0] * (uint64_t)nw;
            } else {
                c0 = col_off[r];
                c1 = col_off[r + 1];
            }
        }
        uint32_t hm = __ballot_sync(0xffffffffu, heavy);
        while (hm) {
            // four records' lines in flight (a record repeats when fewer remain)
            int q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                q[j] = hm ? __ffs(hm) - 1 : q[0];
                if (hm) hm &= hm - 1;
            }
            uint64_t s[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) s[j] = __shfl_sync(0xffffffffu, src, q[j]);
#pragma unroll
            for (int u = 0; u < WPL; ++u) {
                const uint32_t w = lane + 32 * u;
                if (w < nw) acc[u] |= rbits[s[0] + w] | rbits[s[1] + w] | rbits[s[2] + w] | rbits[s[3] + w];
            }
        }
        // light records: their colors laid end to end over the warp, 32 at a
        // time (lane e finds its record by a search over the length prefix)
        const uint32_t len = light ? (uint32_t)(c1 - c0) : 0u;  // < 8192 colors in bitmap mode
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - len;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t e0 = 0; e0 < total; e0 += 32) {
            const uint32_t e = e0 + lane;
            int q = 0;  // the last lane whose range starts at or before e
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const uint32_t ex = __shfl_sync(0xffffffffu, excl, (q + step) & 31);
                if (q + step <= 31 && ex <= e) q += step;
            }
            const uint64_t cq = __shfl_sync(0xffffffffu, c0, q);
            const uint32_t xq = __shfl_sync(0xffffffffu, excl, q);
            if (e < total) {
                const uint32_t v = colors[cq + (e - xq)];
                atomicOr(&bm[v >> 5], 1u << (v & 31));
            }
        }
    }
    __syncwarp();
    uint32_t cnt = 0;
    uint64_t hs = 0;
    uint32_t* out = mbits + m * (uint64_t)nw;
#pragma unroll
    for (int u = 0; u < WPL; ++u) {
        const uint32_t w = lane + 32 * u;
        if (w < nw) {
            const uint32_t x = bm[w] | acc[u];
            out[w] = x;
            cnt += __popc(x);
            if (x) hs += word_mix(w, x);
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    hs = warp_sum64(hs);
    if (lane == 0) {
        msize[m] = cnt;
        mhash[m] = set_hash_final(hs, cnt);
    }
}

// rec_first[r] = smallest node index whose color set is record r's list.
__global__ void k_rec_first(uint64_t D, uint32_t const* __restrict__ n_rec, uint32_t R0,
                            uint32_t* __restrict__ rec_first) {
    uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= D) return;
    const uint32_t r = n_rec[n];
    if (r == NONE32 || (r & MULTI_TAG)) return;
    atomicMin(&rec_first[r - R0], (uint32_t)n);
}

// Candidate class sources: used records then multi nodes.
struct cand_view {
    uint32_t* kind_id;   // record id (global) or MULTI_TAG | m
    uint32_t* first;     // node of first appearance
    uint64_t* hash;
};

__global__ void k_cand_records(uint64_t nrec, uint32_t R0, uint32_t const* __restrict__ rec_first,
                               uint32_t const* __restrict__ keep, uint64_t const* __restrict__ pos,
                               uint64_t const* __restrict__ rhash, cand_view cv, uint32_t* __restrict__ rec_cand) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrec || !keep[i]) return;
    const uint64_t c = pos[i];
    cv.kind_id[c] = R0 + (uint32_t)i;
    cv.first[c] = rec_first[i];
    cv.hash[c] = rhash[R0 + i];
    rec_cand[i] = (uint32_t)c;
}

__global__ void k_cand_multi(uint64_t M, uint64_t base, uint32_t const* __restrict__ mnode,
                             uint64_t const* __restrict__ mhash, cand_view cv) {
    uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    cv.kind_id[base + m] = MULTI_TAG | (uint32_t)m;
    cv.first[base + m] = mnode[m];
    cv.hash[base + m] = mhash[m];
}

struct list_src {
    uint64_t const* col_off;
    uint32_t const* colors;
    uint64_t const* poff;   // list mode: multi-node unions as ascending lists
    uint32_t const* pool;
    uint32_t const* msize;
    uint32_t const* mbits;  // bitmap mode: multi-node unions as C-bit bitmaps
    uint32_t nw;            // 32-bit words per bitmap
};
__device__ __forceinline__ void cand_list(list_src const& L, uint32_t kind_id, uint32_t const*& p, uint64_t& n) {
    if (kind_id & MULTI_TAG) {
        const uint32_t m = kind_id & ~MULTI_TAG;
        p = L.pool ? L.pool + L.poff[m] : nullptr;
        n = L.msize[m];
    } else {
        p = L.colors + L.col_off[kind_id];
        n = L.col_off[kind_id + 1] - L.col_off[kind_id];
    }
}

// A candidate color set: an ascending list, or a bitmap (multi-node unions
// in bitmap mode), with its size.
struct cand_set {
    uint32_t const* list;
    uint32_t const* bm;
    uint64_t n;
};
__device__ __forceinline__ cand_set cand_get(list_src const& L, uint32_t kind_id) {
    cand_set c;
    c.bm = nullptr;
    if ((kind_id & MULTI_TAG) && L.mbits) {
        const uint32_t m = kind_id & ~MULTI_TAG;
        c.list = nullptr;
        c.bm = L.mbits + (uint64_t)m * L.nw;
        c.n = L.msize[m];
        return c;
    }
    cand_list(L, kind_id, c.list, c.n);
    return c;
}
__device__ __forceinline__ cand_set shfl_set(cand_set const& s, int src) {
    cand_set r;
    r.list = (uint32_t const*)__shfl_sync(0xffffffffu, (unsigned long long)s.list, src);
    r.bm = (uint32_t const*)__shfl_sync(0xffffffffu, (unsigned long long)s.bm, src);
    r.n = __shfl_sync(0xffffffffu, (unsigned long long)s.n, src);
    return r;
}

__device__ __forceinline__ bool sets_equal(cand_set const& a, cand_set const& b, uint32_t nw) {
    if (a.n != b.n) return false;
    if (a.bm && b.bm) {
        for (uint32_t w = 0; w < nw; ++w)
            if (a.bm[w] != b.bm[w]) return false;
        return true;
    }
    if (!a.bm && !b.bm) {
        for (uint64_t i = 0; i < a.n; ++i)
            if (a.list[i] != b.list[i]) return false;
        return true;
    }
    // list against bitmap of the same size: equal iff every element is set
    const cand_set& l = a.bm ? b : a;
    const cand_set& m = a.bm ? a : b;
    for (uint64_t i = 0; i < l.n; ++i) {
        const uint32_t v = l.list[i];
        if (!((m.bm[v >> 5] >> (v & 31)) & 1u)) return false;
    }
    return true;
}

// ---- bit ranges -------------------------------------------------------------
__device__ __forceinline__ uint64_t bits_at(uint64_t const* w, uint64_t pos) {
    const uint64_t i = pos >> 6;
    const uint32_t s = (uint32_t)(pos & 63);
    uint64_t v = w[i] >> s;
    if (s) v |= w[i + 1] << (64 - s);
    return v;
}
// Equal bit strings [pa, pa + la) of wa and [pb, pb + lb) of wb.  The hybrid
// encoding is canonical, so equal encodings <=> equal color sets.
__device__ __forceinline__ bool bits_equal(uint64_t const* wa, uint64_t pa, uint64_t la, uint64_t const* wb,
                                           uint64_t pb, uint64_t lb) {
    if (la != lb) return false;
    for (uint64_t i = 0; i < la; i += 64) {
        uint64_t x = bits_at(wa, pa + i) ^ bits_at(wb, pb + i);
        const uint64_t n = la - i;
        if (n < 64) x &= (1ull << n) - 1;
        if (x) return false;
    }
    return true;
}

// ---- hybrid encoding (hybrid_color_sets.hpp:48-95) with the delta code of
// this project's `bits` stand-in: delta(x) = Elias delta of x + 1, LSB-first.
__device__ __forceinline__ uint32_t msb64(uint64_t y) { return 63u - (uint32_t)__clzll((long long)y); }
__device__ __forceinline__ uint32_t delta_bits(uint64_t x) {
    const uint64_t y = x + 1;
    const uint32_t l = msb64(y);
    const uint32_t ll = msb64(l + 1);
    return 2 * ll + 1 + l;
}
__device__ __forceinline__ void or_bits(uint64_t* w, uint64_t pos, uint64_t val, uint32_t len) {
    if (len == 0) return;
    if (len < 64) val &= (1ull << len) - 1;
    const uint64_t i = pos >> 6;
    const uint32_t s = (uint32_t)(pos & 63);
    atomicOr((unsigned long long*)&w[i], (unsigned long long)(val << s));
    if (s && s + len > 64) atomicOr((unsigned long long*)&w[i + 1], (unsigned long long)(val >> (64 - s)));
}
__device__ __forceinline__ uint64_t put_delta(uint64_t* w, uint64_t pos, uint64_t x) {
    const uint64_t y = x + 1;
    const uint32_t l = msb64(y);
    const uint64_t L1 = l + 1;
    const uint32_t ll = msb64(L1);
    // gamma(L1): ll zeros, a one, the low ll bits of L1
    const uint64_t g = (1ull << ll) | ((L1 & ((1ull << ll) - 1)) << (ll + 1));
    or_bits(w, pos, g, 2 * ll + 1);
    pos += 2 * ll + 1;
    if (l) or_bits(w, pos, y, l);
    return pos + l;
}

// One candidate class by the whole warp (bm: the warp's C-bit shared bitmap).
// Pass 0 (ENC = false): encoded size -> nbits[j].  Pass 1: write at bit
// offset pos0 of `words` (zeroed).
template <bool ENC>
__device__ __forceinline__ void encode_one(cand_set const& cs, uint64_t j, uint64_t pos0, uint32_t C, uint32_t nw,
                                           uint32_t* bm, int lane, uint64_t* __restrict__ nbits,
                                           uint64_t* __restrict__ words) {
    const uint64_t N = cs.n;
    const uint64_t sparse_t = (uint64_t)(0.25 * (double)C);
    const uint64_t dense_t = (uint64_t)(0.75 * (double)C);
    const uint32_t hdr = delta_bits(N);
    if (!ENC) {
        // sizes that need no bitmap: the plain-bitmap range has a fixed size,
        // and a sparse set held as an ascending list has its gaps in the list
        if (N >= sparse_t && N < dense_t) {
            if (lane == 0) nbits[j] = hdr + C;
            return;
        }
        if (cs.list && N < sparse_t) {
            uint64_t acc = 0;
            for (uint64_t base = 0; base < N; base += 32) {
                const uint64_t i = base + lane;
                const uint32_t v = i < N ? cs.list[i] : 0u;
                uint32_t pv = __shfl_up_sync(0xffffffffu, v, 1);
                if (lane == 0 && base) pv = cs.list[base - 1];
                if (i < N) acc += delta_bits(i == 0 ? (uint64_t)v : (uint64_t)(v - pv - 1));
            }
            acc = warp_sum64(acc);
            if (lane == 0) nbits[j] = hdr + acc;
            return;
        }
    }
    if (ENC && cs.list && N < sparse_t) {
        // a sparse set held as an ascending list: its gap codes straight
        // from the list, 32 at a time at offsets from a warp scan of their
        // lengths (the codes the bitmap walk below would write)
        if (lane == 0) put_delta(words, pos0, N);
        uint64_t p = pos0 + hdr;
        for (uint64_t base = 0; base < N; base += 32) {
            const uint64_t i = base + lane;
            const uint32_t v = i < N ? cs.list[i] : 0u;
            uint32_t pv = __shfl_up_sync(0xffffffffu, v, 1);
            if (lane == 0 && base) pv = cs.list[base - 1];
            const uint64_t gap = i == 0 ? (uint64_t)v : (uint64_t)(v - pv - 1);
            uint64_t total;
            const uint64_t ex = warp_excl_scan64(i < N ? delta_bits(gap) : 0u, total);
            if (i < N) put_delta(words, p + ex, gap);
            p += total;
        }
        return;
    }
    if (cs.bm) {
        for (uint32_t w = lane; w < nw; w += 32) bm[w] = cs.bm[w];
    } else {
        for (uint32_t w = lane; w < nw; w += 32) bm[w] = 0;
        __syncwarp();
        warp_or_list(bm, cs.list, 0, N, nw, lane);
    }
    __syncwarp();
    uint64_t pos = pos0;
    if (ENC && lane == 0) put_delta(words, pos, N);
    pos += hdr;
    if (N >= sparse_t && N < dense_t) {
        // plain C-bit bitmap
        if (ENC)
            for (uint32_t w = lane; w < nw; w += 32) {
                const uint32_t len = min(32u, C - w * 32);
                or_bits(words, pos + (uint64_t)w * 32, bm[w], len);
            }
        if (!ENC && lane == 0) nbits[j] = hdr + C;
        return;
    }
    const bool want_ones = N < sparse_t;  // else complement: values not in the set
    const uint32_t per = (nw + 31) / 32;
    const uint32_t w0 = lane * per, w1 = min(w0 + per, nw);
    auto word_bits = [&](uint32_t w) -> uint32_t {
        uint32_t x = want_ones ? bm[w] : ~bm[w];
        const uint32_t valid = C - w * 32;
        if (valid < 32) x &= (1u << valid) - 1u;
        return x;
    };
    int32_t last = -1;
    for (uint32_t w = w0; w < w1; ++w) {
        const uint32_t x = word_bits(w);
        if (x) last = (int32_t)(w * 32 + 31 - __clz(x));
    }
    // previous element before this lane's range = max of `last` over lower lanes
    int32_t prev;
    {
        int32_t x = last;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x = max(x, y);
        }
        prev = __shfl_up_sync(0xffffffffu, x, 1);
        if (lane == 0) prev = -1;
    }
    uint64_t mybits = 0;
    {
        int32_t pv = prev;
        for (uint32_t w = w0; w < w1; ++w) {
            uint32_t x = word_bits(w);
            while (x) {
                const uint32_t b = __ffs(x) - 1;
                x &= x - 1;
                const int32_t v = (int32_t)(w * 32 + b);
                mybits += delta_bits(pv < 0 ? (uint64_t)v : (uint64_t)(v - pv - 1));
                pv = v;
            }
        }
    }
    uint64_t total;
    const uint64_t ex = warp_excl_scan64(mybits, total);
    if (!ENC) {
        if (lane == 0) nbits[j] = hdr + total;
        return;
    }
    uint64_t p = pos + ex;
    int32_t pv = prev;
    for (uint32_t w = w0; w < w1; ++w) {
        uint32_t x = word_bits(w);
        while (x) {
            const uint32_t b = __ffs(x) - 1;
            x &= x - 1;
            const int32_t v = (int32_t)(w * 32 + b);
            p = put_delta(words, p, pv < 0 ? (uint64_t)v : (uint64_t)(v - pv - 1));
            pv = v;
        }
    }
}

// Warp per 32 candidate classes: the lanes fetch the 32 candidates' sets
// (and pass-1 offsets) at once, then the warp encodes them one by one, so the
// dependent metadata loads are paid once per 32 candidates.
template <bool ENC>
__global__ void k_encode(uint64_t nc, cand_view cv, list_src L, uint32_t C, uint64_t* __restrict__ nbits,
                         uint64_t const* __restrict__ boff, uint64_t* __restrict__ words) {
    extern __shared__ uint32_t smem_bm[];
    const uint32_t nw = (C + 31) / 32;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* bm = smem_bm + (size_t)wib * nw;
    const uint64_t j0 = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + wib) * 32;
    if (j0 >= nc) return;
    const uint64_t jl = j0 + lane;
    cand_set mine{nullptr, nullptr, 0};
    uint64_t pos = 0;
    if (jl < nc) {
        mine = cand_get(L, cv.kind_id[jl]);
        if (ENC) pos = boff[jl];
    }
    const uint32_t cnt = nc - j0 < 32 ? (uint32_t)(nc - j0) : 32u;
    for (uint32_t q = 0; q < cnt; ++q) {
        const cand_set cs = shfl_set(mine, (int)q);
        const uint64_t p = __shfl_sync(0xffffffffu, pos, (int)q);
        encode_one<ENC>(cs, j0 + q, p, C, nw, bm, lane, nbits, words);
        __syncwarp();  // the next candidate reuses the bitmap
    }
}

// Global class dictionary as seen by kernels: hash slots -> class id, and the
// classes' encodings (bit_off has n + 1 entries).
struct dict_view {
    uint64_t const* slot_hash;
    uint32_t const* slot_cid;
    uint64_t mask;
    uint64_t const* bit_off;
    uint64_t const* words;
};

// Candidate encodings: cw words, cb[c] .. cb[c + 1] bit range of candidate c.
__global__ void k_dict_lookup(uint64_t nc, cand_view cv, uint64_t const* __restrict__ cw,
                              uint64_t const* __restrict__ cb, dict_view D, uint32_t* __restrict__ cid) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const uint64_t h = cv.hash[c];
    uint32_t res = NONE32;
    if (D.slot_hash) {
        uint64_t s = h & D.mask;
        for (uint64_t i = 0; i <= D.mask; ++i) {
            const uint64_t sh = D.slot_hash[s];
            if (sh == HASH_EMPTY) break;
            if (sh == h) {
                const uint32_t k = D.slot_cid[s];
                if (bits_equal(cw, cb[c], cb[c + 1] - cb[c], D.words, D.bit_off[k], D.bit_off[k + 1] - D.bit_off[k])) {
                    res = k;
                    break;
                }
            }
            s = (s + 1) & D.mask;
        }
    }
    cid[c] = res;
}

__global__ void k_new_flags(uint64_t nc, uint32_t const* __restrict__ cid, uint32_t* __restrict__ flag) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) flag[c] = cid[c] == NONE32 ? 1u : 0u;
}

__global__ void k_run_heads(uint64_t n, uint64_t const* __restrict__ key, uint32_t* __restrict__ head) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// run_start[run id] = position of the run's head
__global__ void k_run_starts(uint64_t n, uint32_t const* __restrict__ head, uint64_t const* __restrict__ hpos,
                             uint64_t* __restrict__ run_start) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && head[i]) run_start[hpos[i]] = i;
}

// New class j (in first-appearance order) = candidate rcand[j]; cid base+j.
__global__ void k_assign_new(uint64_t nnew, uint32_t const* __restrict__ rcand, uint64_t base,
                             uint32_t* __restrict__ cid) {
    uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nnew) cid[rcand[j]] = (uint32_t)(base + j);
}

__global__ void k_iota32(uint64_t n, uint32_t* __restrict__ p) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (uint32_t)i;
}

// Set comparison split by length.  A set of at most SHORT_SET words is
// compared by its own lane, eight loads in flight at a time; a longer one by
// the whole warp, lanes reading consecutive words (one coalesced line per
// list per 32 words, four lines in flight per round).
constexpr uint64_t SHORT_SET = 32;

__device__ __forceinline__ uint64_t set_words(cand_set const& a, cand_set const& b, uint32_t nw) {
    return (a.bm && b.bm) ? nw : a.n;
}

// Lane-local equality of two sets of equal size.
__device__ __forceinline__ bool lane_sets_equal(cand_set const& a, cand_set const& b, uint32_t nw) {
    const bool ba = a.bm != nullptr, bb = b.bm != nullptr;
    if (ba == bb) {
        uint32_t const* x = ba ? a.bm : a.list;
        uint32_t const* y = ba ? b.bm : b.list;
        const uint64_t len = ba ? nw : a.n;
        for (uint64_t base = 0; base < len; base += 8) {
            uint32_t u[8], v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = base + q < len;
                u[q] = in ? x[base + q] : 0u;
                v[q] = in ? y[base + q] : 0u;
            }
            bool bad = false;
#pragma unroll
            for (int q = 0; q < 8; ++q) bad |= u[q] != v[q];
            if (bad) return false;
        }
        return true;
    }
    // list against bitmap of the same size: equal iff every element is set
    const cand_set& l = ba ? b : a;
    const cand_set& m = ba ? a : b;
    for (uint64_t base = 0; base < l.n; base += 8) {
        uint32_t u[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) u[q] = base + q < l.n ? l.list[base + q] : NONE32;
        bool bad = false;
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (u[q] != NONE32) bad |= !((m.bm[u[q] >> 5] >> (u[q] & 31)) & 1u);
        if (bad) return false;
    }
    return true;
}

// Warp-wide equality of two sets of equal size (all 32 lanes call it with the
// same arguments).
__device__ __forceinline__ bool warp_sets_equal(cand_set const& a, cand_set const& b, uint32_t nw, int lane) {
    const bool ba = a.bm != nullptr, bb = b.bm != nullptr;
    if (ba == bb) {
        uint32_t const* x = ba ? a.bm : a.list;
        uint32_t const* y = ba ? b.bm : b.list;
        const uint64_t len = ba ? nw : a.n;
        for (uint64_t base = 0; base < len; base += 128) {
            uint32_t u[4], v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint64_t j = base + 32 * q + lane;
                u[q] = j < len ? x[j] : 0u;
                v[q] = j < len ? y[j] : 0u;
            }
            bool bad = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) bad |= u[q] != v[q];
            if (__any_sync(0xffffffffu, bad)) return false;
        }
        return true;
    }
    const cand_set& l = ba ? b : a;
    const cand_set& m = ba ? a : b;
    for (uint64_t base = 0; base < l.n; base += 128) {
        uint32_t u[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint64_t j = base + 32 * q + lane;
            u[q] = j < l.n ? l.list[j] : NONE32;
        }
        bool bad = false;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (u[q] != NONE32) bad |= !((m.bm[u[q] >> 5] >> (u[q] & 31)) & 1u);
        if (__any_sync(0xffffffffu, bad)) return false;
    }
    return true;
}

// Members of an equal-hash run of candidates against the run head, on the
// raw ascending color lists (or bitmaps); rep[c] = head when equal, a
// differing member marks its run for the exact fallback.  Each lane fetches
// its own pair of sets; short pairs are compared by the lane, long ones by
// the warp in turn.  The grid covers n in whole blocks of 256 threads.
__global__ void __launch_bounds__(256) k_member_match_raw(
    uint64_t n, uint32_t const* __restrict__ head, uint64_t const* __restrict__ hpos,
    uint64_t const* __restrict__ run_start, uint32_t const* __restrict__ nidx, cand_view cv, list_src L,
    uint32_t* __restrict__ rep, uint32_t* __restrict__ rep_first, uint32_t* __restrict__ collided) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int need = 0;  // 0: decided, 1: lane compares, 2: warp compares
    bool eq = false;
    uint64_t run = 0;
    uint32_t c = 0, h = 0;
    cand_set sc{nullptr, nullptr, 0}, sh{nullptr, nullptr, 0};
    if (i < n) {
        run = hpos[i] + head[i] - 1;
        c = nidx[i];
        h = nidx[run_start[run]];
        if (c == h) {
            rep[c] = c;
        } else {
            sc = cand_get(L, cv.kind_id[c]);
            sh = cand_get(L, cv.kind_id[h]);
            need = sc.n != sh.n ? 3 : (set_words(sc, sh, L.nw) <= SHORT_SET ? 1 : 2);
        }
    }
    if (need == 1) eq = lane_sets_equal(sc, sh, L.nw);
    uint32_t todo = __ballot_sync(0xffffffffu, need == 2);
    while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const bool e = warp_sets_equal(shfl_set(sc, src), shfl_set(sh, src), L.nw, lane);
        if (lane == src) eq = e;
    }
    if (need) {
        if (eq) {
            rep[c] = h;
        } else {
            rep[c] = c;
            collided[run] = 1;
        }
    }
    // rep_first[h] = min first appearance over the head and its equal
    // members.  A run's positions are consecutive, so the warp takes the
    // minimum per run first and one lane per run issues the atomic: a run of
    // millions of equal sets would otherwise serialize on one address.
    uint32_t f = (i < n && (c == h || eq)) ? cv.first[c] : NONE32;
    const uint64_t key = i < n ? run : ~0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t of = __shfl_down_sync(0xffffffffu, f, o);
        const uint64_t ok = __shfl_down_sync(0xffffffffu, key, o);
        if (lane + o < 32 && ok == key) f = min(f, of);
    }
    const uint64_t pk = __shfl_up_sync(0xffffffffu, key, 1);
    if (i < n && (lane == 0 || pk != key) && f != NONE32) atomicMin(&rep_first[h], f);
}

__global__ void k_group_collided_raw(uint64_t nruns, uint32_t const* __restrict__ collided,
                                     uint64_t const* __restrict__ run_start, uint64_t n,
                                     uint32_t const* __restrict__ nidx, cand_view cv, list_src L,
                                     uint32_t* __restrict__ rep, uint32_t* __restrict__ rep_first) {
    uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns || !collided[r]) return;
    const uint64_t i = run_start[r];
    const uint64_t e = (r + 1 < nruns) ? run_start[r + 1] : n;
    for (uint64_t j = i; j < e; ++j) {
        const uint32_t cj = nidx[j];
        const cand_set sj = cand_get(L, cv.kind_id[cj]);
        uint32_t rr = cj;
        for (uint64_t q = i; q < j; ++q) {
            const uint32_t cq = nidx[q];
            if (rep[cq] != cq) continue;
            if (sets_equal(sj, cand_get(L, cv.kind_id[cq]), L.nw)) {
                rr = cq;
                break;
            }
        }
        rep[cj] = rr;
        const uint32_t f = cv.first[cj];
        if (rr == cj)
            rep_first[cj] = f;
        else if (f < rep_first[rr])
            rep_first[rr] = f;
    }
}

__global__ void k_rep_flags(uint64_t nc, uint32_t const* __restrict__ rep, uint32_t* __restrict__ is_rep) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) is_rep[c] = rep[c] == (uint32_t)c ? 1u : 0u;
}

// Compact the representatives into their own candidate view.
__global__ void k_rep_compact(uint64_t nc, uint32_t const* __restrict__ is_rep, uint64_t const* __restrict__ pos,
                              cand_view cv, uint32_t const* __restrict__ rep_first, cand_view rv,
                              uint32_t* __restrict__ rep_index) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc || !is_rep[c]) return;
    const uint64_t p = pos[c];
    rv.kind_id[p] = cv.kind_id[c];
    rv.first[p] = rep_first[c];
    rv.hash[p] = cv.hash[c];
    rep_index[c] = (uint32_t)p;
}

// New representatives (not in the dictionary): keys = first appearance.
__global__ void k_new_reps(uint64_t nr, uint32_t const* __restrict__ rcid, uint64_t const* __restrict__ npos,
                           cand_view rv, uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nr || rcid[j] != NONE32) return;
    key[npos[j]] = rv.first[j];
    idx[npos[j]] = (uint32_t)j;
}

__global__ void k_cand_cid(uint64_t nc, uint32_t const* __restrict__ rep, uint32_t const* __restrict__ rep_index,
                           uint32_t const* __restrict__ rcid, uint32_t* __restrict__ cid) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) cid[c] = rcid[rep_index[rep[c]]];
}

// Per new class: encoded length, hash and color count (summed per warp,
// one atomic per warp on the shared counter).
__global__ void k_new_sizes(uint64_t nnew, uint32_t const* __restrict__ rcand, cand_view cv, list_src L,
                            uint64_t const* __restrict__ cb, uint64_t* __restrict__ nbits,
                            uint64_t* __restrict__ hashes, unsigned long long* __restrict__ ints) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t n = 0;
    if (j < nnew) {
        const uint32_t c = rcand[j];
        uint32_t const* p;
        cand_list(L, cv.kind_id[c], p, n);
        nbits[j] = cb[c + 1] - cb[c];
        hashes[j] = cv.hash[c];
    }
    const uint64_t sum = warp_sum64(n);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(ints, (unsigned long long)sum);
}

// Append new classes' encodings to the dictionary's bit vector (warp per class;
// words beyond the old end are zero, neighbours share boundary words).
__global__ void k_append_bits(uint64_t nnew, uint32_t const* __restrict__ rcand, uint64_t const* __restrict__ cw,
                              uint64_t const* __restrict__ cb, uint64_t const* __restrict__ dst_off,
                              uint64_t* __restrict__ dw) {
    const uint64_t j = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= nnew) return;
    const uint32_t c = rcand[j];
    const uint64_t a = cb[c], len = cb[c + 1] - a, d = dst_off[j];
    for (uint64_t i = (threadIdx.x & 31) * 64ull; i < len; i += 32 * 64ull) {
        const uint64_t n = len - i < 64 ? len - i : 64;
        or_bits(dw, d + i, bits_at(cw, a + i), (uint32_t)n);
    }
}

__global__ void k_node_cid(uint64_t D, uint32_t const* __restrict__ n_rec, uint32_t R0,
                           uint32_t const* __restrict__ rec_cand, uint64_t mbase, uint32_t const* __restrict__ mgrp,
                           uint32_t const* __restrict__ cid, uint32_t* __restrict__ n_cid) {
    uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= D) return;
    const uint32_t r = n_rec[n];
    uint32_t c = NONE32;
    if (r != NONE32) c = (r & MULTI_TAG) ? cid[mbase + mgrp[r & ~MULTI_TAG]] : cid[rec_cand[r - R0]];
    n_cid[n] = c;
}

// ---- extension masks and clean links -------------------------------------
// Node index of k-mer x, NONE32 when absent.  The tables are read-only once
// the nodes are numbered, so the probes go through the read-only path, and a
// 64-bit-key slot's probe load brings its rank (the node index) along.
// Probes from slot s on: node index of x, or NONE32.
template <typename K>
__device__ __forceinline__ uint32_t node_probe(slot_t<K> const* t, uint32_t cap, uint32_t s, K x) {
    const K EMPTY = kmer_ops<K>::empty();
    for (uint32_t i = 0; i < cap; ++i) {
        slot_t<K> const* e = &t[s];
        if constexpr (sizeof(K) == 8) {
            const ulonglong2 v = __ldg(reinterpret_cast<ulonglong2 const*>(e));
            if (v.x == x) return (uint32_t)v.y;
            if (v.x == EMPTY) return NONE32;
        } else {
            const ulonglong2 kv = __ldg(reinterpret_cast<ulonglong2 const*>(e));
            const K cur = ((u128)kv.y << 64) | (u128)kv.x;
            if (cur == x) return __ldg(&e->rank);
            if (cur == EMPTY) return NONE32;
        }
        s = s + 1 == cap ? 0u : s + 1;
    }
    return NONE32;
}

template <typename K>
__device__ __forceinline__ uint32_t node_lookup(tables<K> const& T, uint32_t tb, K x) {
    const uint32_t cap = (uint32_t)T.tab_cap[tb];
    return node_probe<K>(T.slots + (T.tab_off[tb] - T.off0), cap, slot_of(x, cap), x);
}

// Nodes [*nb, *ne) (one bucket group's, numbered on the device).
// Also records, per side, the node of the neighbour when it is the side's
// only one (link[2n] left, link[2n + 1] right, NONE32 otherwise): k_links
// then needs no probe.
template <typename K>
__global__ void __launch_bounds__(256, 8) k_ext_mask(unsigned long long const* nb, unsigned long long const* ne,
                                                     tables<K> T, K const* __restrict__ n_key,
                                                     uint32_t const* __restrict__ n_bucket, uint32_t k,
                                                     uint8_t* __restrict__ n_mask, uint32_t* __restrict__ link) {
    const uint64_t n = *nb + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= *ne) return;
    typedef kmer_ops<K> ops;
    const K can = n_key[n];
    const K msk = ops::mask(k);
    const K rev = ops::revcomp(can, k);
    const uint32_t tb = n_bucket[n] - T.b0;
    const uint32_t cap = (uint32_t)T.tab_cap[tb];
    slot_t<K> const* t = T.slots + (T.tab_off[tb] - T.off0);
    const uint32_t top = 2 * (k - 1);
    uint32_t out = 0, right = NONE32, left = NONE32;
    // appending nt to x prepends 3 - nt to revcomp(x): (rc(x) >> 2) | (3 - nt) << 2(k-1)
#pragma unroll
    for (uint32_t nt = 0; nt < 4; ++nt) {
        const K hi = (K)(3u - nt) << top;
        const K f = ((can << 2) | (K)nt) & msk;
        const K fr = (rev >> 2) | hi;
        const K cf = f <= fr ? f : fr;
        const uint32_t a = node_probe<K>(t, cap, slot_of(cf, cap), cf);
        if (a != NONE32) {
            out |= 1u << nt;
            right = a;
        }
        const K r = ((rev << 2) | (K)nt) & msk;
        const K rr = (can >> 2) | hi;
        const K cr = r <= rr ? r : rr;
        const uint32_t b = node_probe<K>(t, cap, slot_of(cr, cap), cr);
        if (b != NONE32) {
            out |= 1u << (4 + nt);
            left = b;
        }
    }
    n_mask[n] = (uint8_t)out;
    link[2 * n] = __popc(out >> 4) == 1 ? left : NONE32;
    link[2 * n + 1] = __popc(out & 0xfu) == 1 ? right : NONE32;
}

__device__ __forceinline__ uint32_t fwd_nib(uint32_t m, bool rc) { return (rc ? (m >> 4) : m) & 0xfu; }
__device__ __forceinline__ uint32_t back_nib(uint32_t m, bool rc) { return (rc ? m : (m >> 4)) & 0xfu; }

// link[2n] = L port, link[2n+1] = R port: (node << 1) | rc of the state
// reached, NONE32 when the step is not clean.  On entry link holds the
// sides' only neighbours as k_ext_mask found them.
template <typename K>
__global__ void __launch_bounds__(256, 8) k_links(unsigned long long const* nb, unsigned long long const* ne,
                                                  tables<K> T, K const* __restrict__ n_key,
                                                  uint32_t const* __restrict__ n_bucket,
                                                  uint8_t const* __restrict__ n_mask, uint32_t k,
                                                  uint32_t* __restrict__ link) {
    const uint64_t n = *nb + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= *ne) return;
    typedef kmer_ops<K> ops;
    const K can = n_key[n];
    const uint32_t m = n_mask[n];
    const K msk = ops::mask(k);
    const uint32_t top = 2 * (k - 1);
    const uint32_t nibr = fwd_nib(m, false), nibl = back_nib(m, false);
    const K rev = (__popc(nibr) == 1 || __popc(nibl) == 1) ? ops::revcomp(can, k) : can;
    // R: forward from (can, rc = false)
    uint32_t lr = NONE32, ll = NONE32;
    {
        const uint32_t nib = nibr;
        if (__popc(nib) == 1) {
            const uint32_t nt = __ffs(nib) - 1;
            const K nf = ((can << 2) | (K)nt) & msk;
            const K nr = (rev >> 2) | ((K)(3u - nt) << top);
            const bool nrc = !(nf <= nr);
            const uint32_t nn = link[2 * n + 1];
            if (nn != NONE32 && __popc(back_nib(n_mask[nn], nrc)) == 1) lr = (nn << 1) | (nrc ? 1u : 0u);
        }
    }
    // L: backward from (can, rc = false) = bstep(can, rc = true) then flip
    {
        const uint32_t nib = nibl;
        if (__popc(nib) == 1) {
            const uint32_t nt = __ffs(nib) - 1;
            const K nf = ((rev << 2) | (K)nt) & msk;
            const K nr = (can >> 2) | ((K)(3u - nt) << top);
            const bool srcc = !(nf <= nr);
            const bool nrc = !srcc;
            const uint32_t nn = link[2 * n];
            if (nn != NONE32 && __popc(fwd_nib(n_mask[nn], nrc)) == 1) ll = (nn << 1) | (nrc ? 1u : 0u);
        }
    }
    // a port linked to the node itself ends the chain (the reference's walk
    // meets its own visited k-mer there)
    if (lr != NONE32 && (lr >> 1) == (uint32_t)n) lr = NONE32;
    if (ll != NONE32 && (ll >> 1) == (uint32_t)n) ll = NONE32;
    link[2 * n] = ll;
    link[2 * n + 1] = lr;
}

// ---- chains ---------------------------------------------------------------
struct chain_ws {
    uint32_t const* link;
    uint8_t const* meta;
    uint8_t const* mask;
    uint32_t* ch_node;
    uint8_t* ch_rc;
    unsigned long long* ch_ord;
    uint8_t* ch_vis;
    uint32_t* fe;            // fragment elements (node << 1 | walk rc)
    uint32_t* seed_start;    // per seed node: offset into fe
    uint32_t* seed_len;      // per seed node: elements (0 = not a seed)
    uint8_t* seed_open;
    uint8_t* covered;
    unsigned long long* cursor;
    uint64_t D;
};

// Step forward from state (c, rc): use the R port when rc is false.
__device__ __forceinline__ bool chain_step(uint32_t const* link, uint32_t& c, bool& rc) {
    const uint32_t l = link[2 * (uint64_t)c + (rc ? 0 : 1)];
    if (l == NONE32) return false;
    c = l >> 1;
    rc = ((l & 1u) != 0) != rc;
    return true;
}

__device__ void heap_sort(unsigned long long* a, uint32_t n) {
    auto sift = [&](uint32_t i, uint32_t len) {
        for (;;) {
            uint32_t l = 2 * i + 1, m = i;
            if (l < len && a[l] > a[m]) m = l;
            if (l + 1 < len && a[l + 1] > a[m]) m = l + 1;
            if (m == i) return;
            unsigned long long t = a[i];
            a[i] = a[m];
            a[m] = t;
            i = m;
        }
    };
    if (n < 2) return;
    for (uint32_t i = n / 2; i-- > 0;) sift(i, n);
    for (uint32_t e = n - 1; e > 0; --e) {
        unsigned long long t = a[0];
        a[0] = a[e];
        a[e] = t;
        sift(0, e);
    }
}

// Replay the reference's seed loop on one chain stored at [c0, c0 + L).
__device__ void simulate_chain(chain_ws const& W, uint64_t c0, uint32_t L, bool cyclic) {
    uint32_t const* cn = W.ch_node + c0;
    uint8_t const* crc = W.ch_rc + c0;
    unsigned long long* ord = W.ch_ord + c0;
    uint8_t* vis = W.ch_vis + c0;
    for (uint32_t i = 0; i < L; ++i) {
        ord[i] = ((unsigned long long)cn[i] << 32) | i;
        vis[i] = 0;
    }
    heap_sort(ord, L);
    uint64_t fcur = c0;
    for (uint32_t t = 0; t < L; ++t) {
        const uint32_t p = (uint32_t)(ord[t] & 0xffffffffu);
        if (vis[p]) continue;
        vis[p] = 1;
        const uint32_t s = cn[p];
        const int df = crc[p] ? -1 : 1;  // chain direction of the seed's canonical forward
        const uint32_t sflags = W.meta[s] & 3u;
        uint32_t nb = 0, nf = 0;
        bool open_l = false, open_r = false;
        for (int dir = 0; dir < 2; ++dir) {
            const bool forward = dir == 1;
            if (!forward && sflags == M_LEFT) {
                open_l = __popc(back_nib(W.mask[s], false)) <= 1;
                continue;
            }
            if (forward && sflags == M_RIGHT) {
                open_r = __popc(fwd_nib(W.mask[s], false)) <= 1;
                continue;
            }
            const int step = forward ? df : -df;
            int64_t q = p;
            uint32_t cnt = 0;
            for (;;) {
                int64_t q2 = q + step;
                if (cyclic) {
                    if (q2 < 0) q2 += L;
                    if (q2 >= (int64_t)L) q2 -= L;
                } else if (q2 < 0 || q2 >= (int64_t)L) {
                    break;
                }
                if (vis[q2]) break;
                vis[q2] = 1;
                ++cnt;
                q = q2;
                const uint32_t nd = cn[q];
                const uint32_t f = W.meta[nd] & 3u;
                if (f == M_LEFT || f == M_RIGHT) {
                    const bool wrc = (df == 1) ? (crc[q] != 0) : (crc[q] == 0);
                    if (forward)
                        open_r = __popc(fwd_nib(W.mask[nd], wrc)) <= 1;
                    else
                        open_l = __popc(back_nib(W.mask[nd], wrc)) <= 1;
                    break;
                }
            }
            if (forward)
                nf = cnt;
            else
                nb = cnt;
        }
        const uint32_t flen = nb + 1 + nf;
        for (uint32_t j = 0; j < flen; ++j) {
            int64_t q = (int64_t)p + (int64_t)df * ((int64_t)j - (int64_t)nb);
            if (cyclic) {
                q %= (int64_t)L;
                if (q < 0) q += L;
            }
            const bool wrc = (df == 1) ? (crc[q] != 0) : (crc[q] == 0);
            W.fe[fcur + j] = (cn[q] << 1) | (wrc ? 1u : 0u);
        }
        W.seed_start[s] = (uint32_t)fcur;
        W.seed_len[s] = flen;
        W.seed_open[s] = (uint8_t)((open_l ? 1 : 0) | (open_r ? 2 : 0));
        fcur += flen;
    }
}

// Seed loop of a chain of at most 64 nodes: the visited set is a register
// mask and each seed is the unvisited position with the smallest node index
// (a scan instead of a sort; chains hold one or two fragments in practice).
// Same walk rules as simulate_chain.
__device__ void simulate_chain_small(chain_ws const& W, uint64_t c0, uint32_t L, bool cyclic) {
    uint32_t const* cn = W.ch_node + c0;
    uint8_t const* crc = W.ch_rc + c0;
    const uint64_t all = (L >= 64) ? ~0ull : ((1ull << L) - 1);
    uint64_t vis = 0;
    uint64_t fcur = c0;
    while (vis != all) {
        uint32_t p = 0, best = NONE32;
        for (uint32_t q = 0; q < L; ++q) {
            if ((vis >> q) & 1ull) continue;
            const uint32_t nd = cn[q];
            if (nd < best) {
                best = nd;
                p = q;
            }
        }
        vis |= 1ull << p;
        const uint32_t s = best;
        const int df = crc[p] ? -1 : 1;
        const uint32_t sflags = W.meta[s] & 3u;
        const uint32_t smask = W.mask[s];
        uint32_t nb = 0, nf = 0;
        bool open_l = false, open_r = false;
        for (int dir = 0; dir < 2; ++dir) {
            const bool forward = dir == 1;
            if (!forward && sflags == M_LEFT) {
                open_l = __popc(back_nib(smask, false)) <= 1;
                continue;
            }
            if (forward && sflags == M_RIGHT) {
                open_r = __popc(fwd_nib(smask, false)) <= 1;
                continue;
            }
            const int step = forward ? df : -df;
            int q = (int)p;
            uint32_t cnt = 0;
            for (;;) {
                int q2 = q + step;
                if (cyclic) {
                    if (q2 < 0) q2 += (int)L;
                    if (q2 >= (int)L) q2 -= (int)L;
                } else if (q2 < 0 || q2 >= (int)L) {
                    break;
                }
                if ((vis >> q2) & 1ull) break;
                vis |= 1ull << q2;
                ++cnt;
                q = q2;
                const uint32_t nd = cn[q];
                const uint32_t f = W.meta[nd] & 3u;
                if (f == M_LEFT || f == M_RIGHT) {
                    const bool wrc = (df == 1) ? (crc[q] != 0) : (crc[q] == 0);
                    if (forward)
                        open_r = __popc(fwd_nib(W.mask[nd], wrc)) <= 1;
                    else
                        open_l = __popc(back_nib(W.mask[nd], wrc)) <= 1;
                    break;
                }
            }
            if (forward)
                nf = cnt;
            else
                nb = cnt;
        }
        const uint32_t flen = nb + 1 + nf;
        for (uint32_t j = 0; j < flen; ++j) {
            int q = (int)p + df * ((int)j - (int)nb);
            if (cyclic) {
                q %= (int)L;
                if (q < 0) q += (int)L;
            }
            const bool wrc = (df == 1) ? (crc[q] != 0) : (crc[q] == 0);
            W.fe[fcur + j] = (cn[q] << 1) | (wrc ? 1u : 0u);
        }
        W.seed_start[s] = (uint32_t)fcur;
        W.seed_len[s] = flen;
        W.seed_open[s] = (uint8_t)((open_l ? 1 : 0) | (open_r ? 2 : 0));
        fcur += flen;
    }
}

// Path ends: nodes with at most one linked port, compacted.
__global__ void __launch_bounds__(256) k_chain_ends(chain_ws W, uint32_t* __restrict__ ends,
                                                    unsigned long long* __restrict__ nends) {
    const uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool end = false;
    if (n < W.D) {
        const uint2 l = reinterpret_cast<uint2 const*>(W.link)[n];
        end = (l.x == NONE32) || (l.y == NONE32);
    }
    const unsigned long long at = block_reserve<256>(end ? 1u : 0u, nends);
    if (end) ends[at] = (uint32_t)n;
}

// Each end walks to the other end; the end with the smaller node index leads
// and reserves the chain's slots [c0, c0 + L).  heads[h] = (node | rc << 31,
// L, c0 low, c0 high).
__global__ void __launch_bounds__(256) k_chain_lead(chain_ws W, uint32_t const* __restrict__ ends, uint64_t nends,
                                                    uint4* __restrict__ heads, unsigned long long* __restrict__ nheads,
                                                    uint32_t* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c = 0, L = 0;
    bool rc = false, lead = false;
    if (i < nends) {
        c = ends[i];
        const uint32_t ll = W.link[2 * (uint64_t)c], lr = W.link[2 * (uint64_t)c + 1];
        rc = (lr == NONE32);  // walk out through the linked port
        L = 1;
        lead = true;
        if (ll != NONE32 || lr != NONE32) {
            uint32_t cc = c;
            bool r = rc;
            while (chain_step(W.link, cc, r)) {
                if (++L > W.D) {
                    set_error(err, ERR_CHAIN_LIMIT);
                    lead = false;
                    break;
                }
            }
            if (cc < c) lead = false;  // the other end leads
        }
    }
    const unsigned long long c0 = block_reserve<256>(lead ? L : 0, W.cursor);
    const unsigned long long h = block_reserve<256>(lead ? 1 : 0, nheads);
    if (!lead) return;
    if (c0 + L > W.D) {  // chains partition the nodes; anything else is a bug
        set_error(err, ERR_CAPACITY);
        return;
    }
    heads[h] = make_uint4(c | (rc ? 0x80000000u : 0u), L, (uint32_t)c0, (uint32_t)(c0 >> 32));
}

// One thread per path chain: lay the chain out at c0 and replay the seed loop.
__global__ void __launch_bounds__(128) k_chain_paths(chain_ws W, uint4 const* __restrict__ heads, uint64_t nheads) {
    const uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nheads) return;
    const uint4 hd = heads[h];
    uint32_t cc = hd.x & 0x7fffffffu;
    bool r = (hd.x >> 31) != 0;
    const uint32_t L = hd.y;
    const uint64_t c0 = ((uint64_t)hd.w << 32) | hd.z;
    W.ch_node[c0] = cc;
    W.ch_rc[c0] = r ? 1 : 0;
    W.covered[cc] = 1;
    for (uint32_t i = 1; i < L && chain_step(W.link, cc, r); ++i) {
        W.ch_node[c0 + i] = cc;
        W.ch_rc[c0 + i] = r ? 1 : 0;
        W.covered[cc] = 1;
    }
    if (L <= 64)
        simulate_chain_small(W, c0, L, false);
    else
        simulate_chain(W, c0, L, false);
}

// Cycles: nodes left uncovered; the smallest node index of a cycle leads.
__global__ void k_chain_cycles(chain_ws W, uint32_t* err) {
    uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= W.D || W.covered[n]) return;
    uint32_t cc = (uint32_t)n;
    bool r = false;
    uint32_t L = 1;
    for (;;) {
        if (!chain_step(W.link, cc, r)) {
            set_error(err, ERR_CHAIN_LIMIT);  // an uncovered node must be on a cycle
            return;
        }
        if (cc == n) break;
        if (cc < n) return;
        if (++L > W.D) {
            set_error(err, ERR_CHAIN_LIMIT);
            return;
        }
    }
    const uint64_t c0 = atomicAdd(W.cursor, (unsigned long long)L);
    if (c0 + L > W.D) {
        set_error(err, ERR_CAPACITY);
        return;
    }
    cc = (uint32_t)n;
    r = false;
    W.ch_node[c0] = cc;
    W.ch_rc[c0] = 0;
    for (uint32_t i = 1; i < L; ++i) {
        chain_step(W.link, cc, r);
        W.ch_node[c0 + i] = cc;
        W.ch_rc[c0 + i] = r ? 1 : 0;
    }
    if (L <= 64)
        simulate_chain_small(W, c0, L, true);
    else
        simulate_chain(W, c0, L, true);
}

// ---- fragments --------------------------------------------------------------
__device__ __forceinline__ uint32_t frag_cid(uint32_t const* n_cid, uint32_t node) { return n_cid[node]; }

// Seed nodes in node order (= fragment order): seed_of[f] = node of fragment f.
__global__ void k_seed_flags(uint64_t D, uint32_t const* __restrict__ seed_len, uint32_t* __restrict__ is_seed) {
    uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n < D) is_seed[n] = seed_len[n] ? 1u : 0u;
}
__global__ void k_seed_list(uint64_t D, uint32_t const* __restrict__ is_seed, uint64_t const* __restrict__ fpos,
                            uint32_t* __restrict__ seed_of) {
    uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n < D && is_seed[n]) seed_of[fpos[n]] = (uint32_t)n;
}

// Thread per fragment: serialized size (frag_unitig_writer::write_batch layout).
__global__ void k_frag_sizes(uint64_t F, uint32_t const* __restrict__ seed_of, uint32_t const* __restrict__ seed_start,
                             uint32_t const* __restrict__ seed_len, uint32_t const* __restrict__ fe,
                             uint32_t const* __restrict__ n_cid, uint32_t k, uint64_t* __restrict__ sz,
                             unsigned long long* __restrict__ seq_total) {
    uint64_t f = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t seq = 0;
    if (f < F) {
        const uint32_t n = seed_of[f];
        const uint32_t len = seed_len[n], a = seed_start[n];
        uint32_t runs = 1, prev = frag_cid(n_cid, fe[a] >> 1);
        for (uint32_t j = 1; j < len; ++j) {
            const uint32_t c = frag_cid(n_cid, fe[a + j] >> 1);
            runs += c != prev;
            prev = c;
        }
        seq = (uint64_t)k + len - 1;
        sz[f] = 1 + 4 + 12ull * runs + 4 + seq;
    }
    seq = prim::warp_inclusive_scan(seq);
    if ((threadIdx.x & 31) == 31 && seq) atomicAdd(seq_total, (unsigned long long)seq);
}

__device__ __forceinline__ void put_bytes(uint8_t* o, uint64_t v, int n) {
    for (int i = 0; i < n; ++i) o[i] = (uint8_t)(v >> (8 * i));
}

// One fragment record (unitig_spill.hpp:491-522 layout) at `o` (shared or
// global memory).  Each base after the first k-mer is the last base of the
// oriented k-mer: the low 2 bits of the key, or the complement of its first
// base when the walk is reverse -- no reverse complement per element.
template <typename K>
__device__ __forceinline__ void emit_fragment(uint8_t* o, uint32_t n, uint32_t const* __restrict__ seed_start,
                                              uint32_t const* __restrict__ seed_len,
                                              uint8_t const* __restrict__ seed_open, uint32_t const* __restrict__ fe,
                                              uint32_t const* __restrict__ n_cid, K const* __restrict__ n_key,
                                              uint32_t k) {
    typedef kmer_ops<K> ops;
    const uint32_t len = seed_len[n];
    const uint32_t a = seed_start[n];
    o[0] = seed_open[n];
    uint32_t runs = 0;
    uint8_t* rp = o + 5;
    uint32_t prev = frag_cid(n_cid, fe[a] >> 1), cnt = 1;
    for (uint32_t j = 1; j <= len; ++j) {
        const uint32_t c = j < len ? frag_cid(n_cid, fe[a + j] >> 1) : ~prev;
        if (j < len && c == prev) {
            ++cnt;
            continue;
        }
        const uint64_t cid64 = prev == NONE32 ? ~0ull : (uint64_t)prev;
        put_bytes(rp, cid64, 8);
        put_bytes(rp + 8, cnt, 4);
        rp += 12;
        ++runs;
        prev = c;
        cnt = 1;
    }
    put_bytes(o + 1, runs, 4);
    const uint32_t seq_len = k + len - 1;
    put_bytes(rp, seq_len, 4);
    uint8_t* sp = rp + 4;
    const char acgt[4] = {'A', 'C', 'G', 'T'};
    {
        const uint32_t e = fe[a];
        K w = n_key[e >> 1];
        if (e & 1u) w = ops::revcomp(w, k);
        for (uint32_t i = 0; i < k; ++i) sp[k - 1 - i] = acgt[ops::low2(w >> (2 * i))];
    }
    const uint32_t top = 2 * (k - 1);
    for (uint32_t j = 1; j < len; ++j) {
        const uint32_t e = fe[a + j];
        const K w = n_key[e >> 1];
        const uint32_t b = (e & 1u) ? 3u - ops::low2(w >> top) : ops::low2(w);
        sp[k - 1 + j] = acgt[b];
    }
}

// Fragments [f0, f0 + FW_THREADS) of a block occupy one contiguous byte range
// of the output.  They are laid out in shared memory with the range's
// 16-byte phase and stored with aligned 16-byte writes (bytes at the two
// ragged ends one by one), instead of a few dozen scattered byte stores per
// fragment.  A block whose range does not fit writes directly.
constexpr int FW_THREADS = 128;
constexpr int FW_BYTES = 32 * 1024;

template <typename K>
__global__ void __launch_bounds__(FW_THREADS)
    k_frag_write(uint64_t F, uint32_t const* __restrict__ seed_of, uint32_t const* __restrict__ seed_start,
                 uint32_t const* __restrict__ seed_len, uint8_t const* __restrict__ seed_open,
                 uint32_t const* __restrict__ fe, uint32_t const* __restrict__ n_cid, K const* __restrict__ n_key,
                 uint32_t k, uint64_t const* __restrict__ off, uint8_t* __restrict__ out) {
    __shared__ __align__(16) uint8_t buf[FW_BYTES];
    const uint64_t f0 = (uint64_t)blockIdx.x * FW_THREADS;
    const uint64_t f1 = (f0 + FW_THREADS < F) ? f0 + FW_THREADS : F;
    const uint64_t g0 = off[f0], g1 = off[f1];
    const uint32_t phase = (uint32_t)(g0 & 15);
    const uint64_t f = f0 + threadIdx.x;
    if (g1 - g0 + phase > (uint64_t)FW_BYTES) {  // block-uniform
        if (f < F) emit_fragment<K>(out + off[f], seed_of[f], seed_start, seed_len, seed_open, fe, n_cid, n_key, k);
        return;
    }
    if (f < F)
        emit_fragment<K>(buf + phase + (off[f] - g0), seed_of[f], seed_start, seed_len, seed_open, fe, n_cid, n_key,
                         k);
    __syncthreads();
    const uint64_t a0 = (g0 + 15) & ~uint64_t(15);  // first aligned byte inside the range
    const uint64_t a1 = g1 & ~uint64_t(15);         // end of the aligned part
    if (a0 >= a1) {
        for (uint64_t b = g0 + threadIdx.x; b < g1; b += FW_THREADS) out[b] = buf[phase + (b - g0)];
        return;
    }
    for (uint64_t b = g0 + threadIdx.x; b < a0; b += FW_THREADS) out[b] = buf[phase + (b - g0)];
    for (uint64_t b = a1 + threadIdx.x; b < g1; b += FW_THREADS) out[b] = buf[phase + (b - g0)];
    const uint64_t nchunks = (a1 - a0) >> 4;
    uint4 const* src = reinterpret_cast<uint4 const*>(buf + phase + (a0 - g0));  // 16-byte aligned
    uint4* dst = reinterpret_cast<uint4*>(out + a0);
    for (uint64_t c = threadIdx.x; c < nchunks; c += FW_THREADS) dst[c] = src[c];
}

// ---------------------------------------------------------------------------
// ---- small helpers ----------------------------------------------------------
__global__ void k_count_flags(uint64_t n, uint32_t const* __restrict__ f, unsigned long long* __restrict__ c) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t v = (i < n) ? f[i] : 0u;
    const uint32_t b = __ballot_sync(0xffffffffu, v != 0);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(c, (unsigned long long)__popc(b));
}
__global__ void k_add_offsets(uint64_t n, uint64_t const* __restrict__ src, uint64_t add,
                              uint64_t* __restrict__ dst) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i] + add;
}
__global__ void k_set_u64(uint64_t* p, uint64_t v) { *p = v; }
__global__ void k_copy_u64(unsigned long long const* src, unsigned long long* dst) { *dst = *src; }
__global__ void k_used_flags(uint64_t n, uint32_t const* __restrict__ first, uint32_t* __restrict__ keep) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keep[i] = first[i] != NONE32 ? 1u : 0u;
}

void add_offsets(uint64_t const* src, uint64_t n, uint64_t add, uint64_t* dst, cudaStream_t st) {
    if (!n) return;
    k_add_offsets<<<grid(n, 256), 256, 0, st>>>(n, src, add, dst);
    CDBG_CHECK_LAUNCH();
}

void check_device_error_word(uint32_t* d_err, cudaStream_t st, char const* stage) {
    const uint32_t e = read_dev(d_err, st);
    if (e == ERR_NONE) return;
    CDBG_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    static char const* names[] = {"none", "hash table full", "field overflow", "malformed record",
                                  "capacity exceeded", "chain walk bound exceeded"};
    throw std::runtime_error(std::string("device error in ") + stage + ": " +
                             (e < 6 ? names[e] : "unknown"));
}

// ---------------------------------------------------------------------------
__global__ void k_dict_insert(uint64_t c0, uint64_t c1, uint64_t const* __restrict__ cls_hash,
                              uint64_t* __restrict__ slot_hash, uint32_t* __restrict__ slot_cid, uint64_t mask,
                              uint32_t* err) {
    uint64_t c = c0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    const uint64_t h = cls_hash[c];
    uint64_t s = h & mask;
    for (uint64_t i = 0; i <= mask; ++i) {
        const uint64_t old = atomicCAS((unsigned long long*)&slot_hash[s], (unsigned long long)HASH_EMPTY,
                                       (unsigned long long)h);
        if (old == HASH_EMPTY) {
            slot_cid[s] = (uint32_t)c;
            return;
        }
        s = (s + 1) & mask;
    }
    set_error(err, ERR_TABLE_FULL);
}

// Global color-class dictionary (persists across bucket batches): per class
// its 64-bit set hash and its bit range in the encoded .color_sets vector; an
// open-addressing table hash -> class id.  Equality is tested on encodings.
struct class_dict {
    dvec<uint64_t>& cls_hash;  // n
    dvec<uint64_t>& bit_off;   // n + 1 (last = nbits)
    dvec<uint64_t>& words;     // encoded classes, zero beyond nbits
    dvec<uint64_t>& slot_hash;
    dvec<uint32_t>& slot_cid;
    uint64_t n = 0, nbits = 0, total_integers = 0, mask = 0;

    explicit class_dict(phase2_state& S)
        : cls_hash(S.cls_hash), bit_off(S.bit_off), words(S.words), slot_hash(S.slot_hash), slot_cid(S.slot_cid) {}

    // Start empty, keeping the storage of a previous build (words are zeroed
    // where the previous build wrote).
    void init(cudaStream_t st) {
        bit_off.reserve(1024, st);
        CDBG_CUDA(cudaMemsetAsync(bit_off.p, 0, 8, st));
        bit_off.n = 1;
        words.reserve(1024, st, true);
        if (words.n) CDBG_CUDA(cudaMemsetAsync(words.p, 0, 8 * std::min(words.n + 4, words.cap), st));
        words.n = 0;
        cls_hash.n = 0;
    }
    dict_view view() const { return dict_view{slot_hash.p, slot_cid.p, mask, bit_off.p, words.p}; }
    // Make room for n classes (load <= 1/2); classes [first_new, n) still need
    // inserting.  A resized table is rebuilt from every class hash.
    void ensure_table(uint64_t first_new, cudaStream_t st, uint32_t* d_err) {
        uint64_t cap = 1024;
        while (cap < 2 * n) cap <<= 1;
        uint64_t from = first_new;
        if (!slot_hash.p || cap - 1 > mask) {
            slot_hash.reserve(cap, st);
            slot_cid.reserve(cap, st);
            mask = cap - 1;
            CDBG_CUDA(cudaMemsetAsync(slot_hash.p, 0xff, cap * 8, st));
            from = 0;
        }
        if (n > from) {
            k_dict_insert<<<grid(n - from, 256), 256, 0, st>>>(from, n, cls_hash.p, slot_hash.p, slot_cid.p, mask,
                                                              d_err);
            CDBG_CHECK_LAUNCH();
        }
    }
};

template <typename K>
void run_batch(record_set const& rs, rec_view const& R, phase2_params const& p, uint32_t b0, uint32_t b1,
               std::vector<uint64_t> const& bocc, dev_arena& A, cudaStream_t st, uint32_t* d_err,
               class_dict& dict, phase2_result& out, std::vector<uint64_t> const& hbstart, uint64_t* d_rhash,
               dvec<uint8_t>& dfrag, dvec<uint64_t>& dfoff) {
    const uint32_t k = p.k, C = p.num_colors;
    const uint64_t R0 = hbstart[b0], R1 = hbstart[b1];
    const uint64_t nrec = R1 - R0;
    const uint64_t O0 = bocc[b0], O1 = bocc[b1];
    const uint64_t nocc = O1 - O0;
    if (nocc == 0) return;
    auto mark = A.mark();
    // ---- tables: one open-addressing table per bucket, processed in bucket
    // groups of at most p.group_bytes of tables (one group per batch by
    // default): a group's tables are built, numbered and probed (insert, first
    // occurrences, nodes, extension masks, links) before the next group
    // reuses their memory, so a group that fits in L2 stays cache-resident
    const uint32_t nb = b1 - b0;
    const uint64_t q = std::min<uint32_t>(16, std::max<uint32_t>(5, p.table_slots_q));
    std::vector<uint64_t> toff(nb + 1), tcap(nb);
    uint64_t T = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint64_t o = bocc[b0 + b + 1] - bocc[b0 + b];
        // slots per occurrence q/4 > 1 (distinct <= occurrences): the default
        // 2 keeps the load factor <= 1/2 for short unsuccessful probes in the
        // neighbour lookups
        const uint64_t cap = o ? std::max<uint64_t>(64, (o * q + 3) / 4 + 16) : 0;
        toff[b] = T;
        tcap[b] = cap;
        T += cap;
    }
    toff[nb] = T;
    if (T >= (1ull << 31)) throw std::runtime_error("k-mer table of one bucket batch exceeds 2^31 slots");
    if (nrec > MAX_BATCH_RECORDS) throw std::runtime_error("more than 2^28 - 2 records in one bucket");
    const uint64_t gslots = std::max<uint64_t>(1024, p.group_bytes / sizeof(slot_t<K>));
    std::vector<uint32_t> gb{0};  // group boundaries (batch-relative buckets)
    for (uint32_t b = 1; b <= nb; ++b)
        if (b == nb || toff[b + 1] - toff[gb.back()] > gslots) gb.push_back(b);
    if (gb.back() != nb) gb.push_back(nb);
    const size_t ng = gb.size() - 1;
    uint64_t Tmax = 0;
    for (size_t g = 0; g < ng; ++g) Tmax = std::max<uint64_t>(Tmax, toff[gb[g + 1]] - toff[gb[g]]);
    uint32_t* occ_slot = A.alloc<uint32_t>(nocc);
    uint64_t* d_toff = A.alloc<uint64_t>(nb + 1);
    uint64_t* d_tcap = A.alloc<uint64_t>(nb);
    CDBG_CUDA(cudaMemcpyAsync(d_toff, toff.data(), 8ull * (nb + 1), cudaMemcpyHostToDevice, st));
    CDBG_CUDA(cudaMemcpyAsync(d_tcap, tcap.data(), 8ull * nb, cudaMemcpyHostToDevice, st));
    slot_t<K>* slots = A.alloc<slot_t<K>>(Tmax + 1);
    // record of each occurrence block's first occurrence (k_insert, k_multi_pairs)
    const uint64_t nblk = ceil_div(nocc, (uint64_t)OCC_BLOCK);
    uint32_t* blk_rec = A.alloc<uint32_t>(nblk + 1);
    k_block_records<<<grid(nrec, 256), 256, 0, st>>>(R.occ, R0, nrec, O0, nblk, blk_rec);
    CDBG_CHECK_LAUNCH();
    const uint64_t nwb = ceil_div(nocc, 32);
    uint32_t* bits = A.alloc<uint32_t>(nwb);
    CDBG_CUDA(cudaMemsetAsync(bits, 0, 4 * nwb, st));
    // node arrays, sized for the worst case (every occurrence a distinct
    // k-mer): the groups number their nodes on the device, without a host
    // round trip per group
    K* n_key = A.alloc<K>(nocc);
    uint8_t* n_meta = A.alloc<uint8_t>(nocc);
    uint32_t* n_rec = A.alloc<uint32_t>(nocc);
    uint32_t* n_bucket = A.alloc<uint32_t>(nocc);
    uint8_t* n_mask = A.alloc<uint8_t>(nocc);
    uint32_t* link = A.alloc<uint32_t>(2 * nocc);
    // look-back state of every group's numbering, zeroed once
    std::vector<uint64_t> gtile(ng + 1, 0);
    for (size_t g = 0; g < ng; ++g)
        gtile[g + 1] = gtile[g] + ceil_div(bocc[b0 + gb[g + 1]] - bocc[b0 + gb[g]], (uint64_t)MN_ROUNDS * 256);
    unsigned long long* mn_status = A.alloc<unsigned long long>(gtile[ng] + 1);
    uint32_t* mn_counter = A.alloc<uint32_t>(ng + 1);
    unsigned long long* ncnt = A.alloc<unsigned long long>(2);  // node bases, alternating by group
    CDBG_CUDA(cudaMemsetAsync(mn_status, 0, 8 * (gtile[ng] + 1), st));
    CDBG_CUDA(cudaMemsetAsync(mn_counter, 0, 4 * (ng + 1), st));
    CDBG_CUDA(cudaMemsetAsync(ncnt, 0, 16, st));
    for (size_t g = 0; g < ng; ++g) {
        const uint32_t g0 = gb[g], g1 = gb[g + 1];
        const uint64_t t0 = bocc[b0 + g0] - O0, tn = bocc[b0 + g1] - bocc[b0 + g0];
        const uint64_t Tg = toff[g1] - toff[g0];
        if (tn == 0) {
            // no occurrence: the next group starts from the same node count
            k_copy_u64<<<1, 1, 0, st>>>(ncnt + (g & 1), ncnt + ((g + 1) & 1));
            CDBG_CHECK_LAUNCH();
            continue;
        }
        tables<K> TG;
        TG.slots = slots;
        TG.tab_off = d_toff + g0;
        TG.tab_cap = d_tcap + g0;
        TG.b0 = b0 + g0;
        TG.off0 = toff[g0];
        {
            CDBG_PROF("k_init_tables", st);
            k_init_tables<K><<<grid(Tg, 256), 256, 0, st>>>(Tg, slots);
        }
        CDBG_CHECK_LAUNCH();
        {
            CDBG_PROF("k_insert", st);
            k_insert<K><<<grid(tn, 256), 256, 0, st>>>(R, TG, R0, nrec, O0, t0, tn, k, blk_rec, occ_slot, d_err);
        }
        CDBG_CHECK_LAUNCH();
        {
            CDBG_PROF("k_firstbits", st);
            k_firstbits<K><<<grid(Tg, 256), 256, 0, st>>>(Tg, slots, bits);
        }
        CDBG_CHECK_LAUNCH();
        unsigned long long* nbase = ncnt + (g & 1);
        unsigned long long* nnext = ncnt + ((g + 1) & 1);
        {
            CDBG_PROF("k_make_nodes", st);
            k_make_nodes<K><<<(unsigned)(gtile[g + 1] - gtile[g]), 256, 0, st>>>(
                t0, tn, occ_slot, bits, TG, g1 - g0, R0, nbase, nnext, mn_counter + g, mn_status + gtile[g],
                n_key, n_meta, n_rec, n_bucket, d_err);
        }
        CDBG_CHECK_LAUNCH();
        {
            CDBG_PROF("k_ext_mask", st);
            k_ext_mask<K><<<grid(tn, 256), 256, 0, st>>>(nbase, nnext, TG, n_key, n_bucket, k, n_mask, link);
        }
        CDBG_CHECK_LAUNCH();
        {
            CDBG_PROF("k_links", st);
            k_links<K><<<grid(tn, 256), 256, 0, st>>>(nbase, nnext, TG, n_key, n_bucket, n_mask, k, link);
        }
        CDBG_CHECK_LAUNCH();
        if (ng > 1) {
            // the next group reuses this group's table memory: occurrences
            // keep their node index instead of their slot
            {
                CDBG_PROF("k_occ_nodes", st);
                k_occ_nodes<K><<<grid(tn, 256), 256, 0, st>>>(t0, tn, occ_slot, slots, toff[g0]);
            }
            CDBG_CHECK_LAUNCH();
        }
    }
    const uint64_t D = read_dev(ncnt + (ng & 1), st);
    if (D >= (1ull << 31)) throw std::runtime_error("too many distinct k-mers in one bucket batch");
    check_device_error_word(d_err, st, "k-mer table insert");
    // ---- multi-record k-mers: (node, record) pairs in one pass, at most one
    // per occurrence
    unsigned long long* cnt = A.alloc<unsigned long long>(1);
    uint32_t* tile_counter = A.alloc<uint32_t>(1);
    const uint64_t mp_tiles = ceil_div(nblk, (uint64_t)MP_ROUNDS);
    unsigned long long* status = A.alloc<unsigned long long>(mp_tiles);
    uint32_t* pnode = A.alloc<uint32_t>(nocc);
    uint32_t* prec = A.alloc<uint32_t>(nocc);
    CDBG_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
    CDBG_CUDA(cudaMemsetAsync(tile_counter, 0, 4, st));
    CDBG_CUDA(cudaMemsetAsync(status, 0, 8 * mp_tiles, st));
    {
        CDBG_PROF("k_multi_pairs", st);
        // one group: the table is still whole, and an occurrence's slot holds
        // its node index (rank field); several: occ_slot holds node indices
        uint32_t const* rankp = ng == 1 ? reinterpret_cast<uint32_t const*>(
                                              reinterpret_cast<char const*>(slots) + offsetof(slot_t<K>, rank))
                                        : nullptr;
        k_multi_pairs<<<(unsigned)mp_tiles, OCC_BLOCK, 0, st>>>(R.occ, R0, nrec, O0, nocc, blk_rec, occ_slot,
                                                            rankp, (uint32_t)(sizeof(slot_t<K>) / 4), n_rec,
                                                            tile_counter, status, cnt, pnode, prec, nocc, d_err);
    }
    CDBG_CHECK_LAUNCH();
    const uint64_t npairs = read_dev(cnt, st);
    uint64_t M = 0;
    uint32_t* mnode = nullptr;
    uint64_t* moff = nullptr;
    uint64_t* upairs = nullptr;
    uint32_t* msize = nullptr;
    uint64_t* mhash = nullptr;
    uint64_t* poff = nullptr;
    uint32_t* pool = nullptr;
    uint32_t* mbits = nullptr;
    uint64_t G = 0;              // union groups
    uint32_t* gnode = nullptr;   // first node of each group
    uint64_t* gbeg = nullptr;    // record range of each group
    uint64_t* gend = nullptr;
    uint32_t* mgrp = nullptr;    // group of each multi node
    if (npairs) {
        // stable by node (records already ascend within a node): the node bits only
        const int node_bits = D > 1 ? 64 - __builtin_clzll(D - 1) : 1;
        prim::radix_sort_pairs<uint32_t, uint32_t>(pnode, prec, npairs, 0, node_bits, A, st, d_err);
        uint32_t* keep = A.alloc<uint32_t>(npairs);
        uint64_t* kpos = A.alloc<uint64_t>(npairs + 1);
        k_unique_pairs<<<grid(npairs, 256), 256, 0, st>>>(npairs, pnode, prec, keep);
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(keep, kpos, npairs, A, st, kpos + npairs);
        const uint64_t nu = read_dev(kpos + npairs, st);
        upairs = A.alloc<uint64_t>(nu);
        k_compact_pairs<<<grid(npairs, 256), 256, 0, st>>>(npairs, pnode, prec, keep, kpos, upairs);
        CDBG_CHECK_LAUNCH();
        uint32_t* head = A.alloc<uint32_t>(nu);
        uint64_t* hpos = A.alloc<uint64_t>(nu + 1);
        k_node_heads<<<grid(nu, 256), 256, 0, st>>>(nu, upairs, head);
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(head, hpos, nu, A, st, hpos + nu);
        M = read_dev(hpos + nu, st);
        mnode = A.alloc<uint32_t>(M);
        moff = A.alloc<uint64_t>(M + 1);
        k_multi_index<<<grid(nu, 256), 256, 0, st>>>(nu, upairs, head, hpos, mnode, moff, n_rec);
        CDBG_CHECK_LAUNCH();
        k_set_u64<<<1, 1, 0, st>>>(moff + M, nu);
        CDBG_CHECK_LAUNCH();
        // one union per run of multi nodes with the same owning records
        {
            uint32_t* ghead = A.alloc<uint32_t>(M);
            uint64_t* gpos = A.alloc<uint64_t>(M + 1);
            k_multi_same<<<grid(M, 256), 256, 0, st>>>(M, moff, upairs, ghead);
            CDBG_CHECK_LAUNCH();
            prim::exclusive_scan<uint32_t, uint64_t>(ghead, gpos, M, A, st, gpos + M);
            G = read_dev(gpos + M, st);
            gnode = A.alloc<uint32_t>(G);
            gbeg = A.alloc<uint64_t>(G);
            gend = A.alloc<uint64_t>(G);
            mgrp = A.alloc<uint32_t>(M);
            k_multi_groups<<<grid(M, 256), 256, 0, st>>>(M, ghead, gpos, mnode, moff, gnode, gbeg, gend, mgrp);
            CDBG_CHECK_LAUNCH();
        }
        msize = A.alloc<uint32_t>(G);
        mhash = A.alloc<uint64_t>(G);
        const uint32_t nw = (C + 31) / 32;
        int wpb = (int)std::max<uint64_t>(1, std::min<uint64_t>(8, (96 * 1024) / (4ull * nw)));
        const size_t shm = (size_t)wpb * nw * 4;
        if (p.union_bitmaps) {
            // heavy records (>= 64 colors) used by multi-record nodes get a bitmap once
            uint32_t* hflag = A.alloc<uint32_t>(nrec);
            uint64_t* hpos = A.alloc<uint64_t>(nrec + 1);
            CDBG_CUDA(cudaMemsetAsync(hflag, 0, 4 * nrec, st));
            k_heavy_flags<<<grid(nu, 256), 256, 0, st>>>(nu, upairs, R.col_off, (uint32_t)R0,
                                                          std::max<uint32_t>(1, p.heavy_colors), hflag);
            CDBG_CHECK_LAUNCH();
            prim::exclusive_scan<uint32_t, uint64_t>(hflag, hpos, nrec, A, st, hpos + nrec);
            const uint64_t nheavy = read_dev(hpos + nrec, st);
            uint32_t* rbits = A.alloc<uint32_t>(nheavy * nw + 1);
            if (shm > 48 * 1024)
                CDBG_CUDA(cudaFuncSetAttribute(k_heavy_bitmaps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
            if (nheavy) {
                CDBG_PROF("k_heavy_bitmaps", st);
                k_heavy_bitmaps<<<grid(ceil_div(nrec, 32), wpb), wpb * 32, shm, st>>>(nrec, hflag, hpos, (uint32_t)R0, R.col_off,
                                                                        R.colors, nw, rbits);
            }
            CDBG_CHECK_LAUNCH();
            mbits = A.alloc<uint32_t>(G * nw + 1);
            {
                CDBG_PROF("k_union", st);
                auto launch = [&](auto kern) {
                    if (shm > 48 * 1024)
                        CDBG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
                    kern<<<grid(G, wpb), wpb * 32, shm, st>>>(G, gbeg, gend, upairs, R.col_off, R.colors, (uint32_t)R0,
                                                              hflag, hpos, rbits, nw, mbits, msize, mhash);
                };
                if (nw <= 32)
                    launch(k_union_bm<1>);
                else if (nw <= 64)
                    launch(k_union_bm<2>);
                else if (nw <= 128)
                    launch(k_union_bm<4>);
                else if (nw <= 256)
                    launch(k_union_bm<8>);
                else
                    throw std::runtime_error("bitmap unions need at most 8192 colors");
            }
            CDBG_CHECK_LAUNCH();
        } else {
            if (shm > 48 * 1024) {
                CDBG_CUDA(cudaFuncSetAttribute(k_union<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
                CDBG_CUDA(cudaFuncSetAttribute(k_union<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
            }
            {
                CDBG_PROF("k_union", st);
                k_union<false><<<grid(G, wpb), wpb * 32, shm, st>>>(G, gbeg, gend, upairs, R.col_off, R.colors, C,
                                                                     msize, mhash, nullptr, nullptr);
            }
            CDBG_CHECK_LAUNCH();
            poff = A.alloc<uint64_t>(G + 1);
            prim::exclusive_scan<uint32_t, uint64_t>(msize, poff, G, A, st, poff + G);
            const uint64_t ptot = read_dev(poff + G, st);
            pool = A.alloc<uint32_t>(ptot + 1);
            {
                CDBG_PROF("k_union", st);
                k_union<true><<<grid(G, wpb), wpb * 32, shm, st>>>(G, gbeg, gend, upairs, R.col_off, R.colors, C,
                                                                    msize, mhash, poff, pool);
            }
            CDBG_CHECK_LAUNCH();
        }
    }
    out.n_multi += M;
    // ---- candidates: used records, then multi nodes
    uint32_t* rec_first = A.alloc<uint32_t>(nrec);
    CDBG_CUDA(cudaMemsetAsync(rec_first, 0xff, 4 * nrec, st));
    {
        CDBG_PROF("k_rec_first", st);
        k_rec_first<<<grid(D, 256), 256, 0, st>>>(D, n_rec, (uint32_t)R0, rec_first);
    }
    CDBG_CHECK_LAUNCH();
    uint32_t* rkeep = A.alloc<uint32_t>(nrec);
    uint64_t* rpos = A.alloc<uint64_t>(nrec + 1);
    k_used_flags<<<grid(nrec, 256), 256, 0, st>>>(nrec, rec_first, rkeep);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint32_t, uint64_t>(rkeep, rpos, nrec, A, st, rpos + nrec);
    const uint64_t nrc = read_dev(rpos + nrec, st);
    const uint64_t nc = nrc + G;
    cand_view cv;
    cv.kind_id = A.alloc<uint32_t>(nc + 1);
    cv.first = A.alloc<uint32_t>(nc + 1);
    cv.hash = A.alloc<uint64_t>(nc + 1);
    uint32_t* rec_cand = A.alloc<uint32_t>(nrec);
    k_cand_records<<<grid(nrec, 256), 256, 0, st>>>(nrec, (uint32_t)R0, rec_first, rkeep, rpos, d_rhash, cv, rec_cand);
    CDBG_CHECK_LAUNCH();
    if (G) {
        k_cand_multi<<<grid(G, 256), 256, 0, st>>>(G, nrc, gnode, mhash, cv);
        CDBG_CHECK_LAUNCH();
    }
    list_src L{R.col_off, R.colors, poff, pool, msize, mbits, (C + 31) / 32};
    uint32_t* cid = A.alloc<uint32_t>(nc + 1);
    if (nc) {
        // 1. group candidates with equal color sets (sort by set hash, then
        //    compare raw lists inside equal-hash runs)
        uint64_t* skey = A.alloc<uint64_t>(nc);
        uint32_t* sidx = A.alloc<uint32_t>(nc);
        CDBG_CUDA(cudaMemcpyAsync(skey, cv.hash, 8 * nc, cudaMemcpyDeviceToDevice, st));
        k_iota32<<<grid(nc, 256), 256, 0, st>>>(nc, sidx);
        CDBG_CHECK_LAUNCH();
        prim::sort_pairs_u64_exact<uint32_t>(skey, sidx, nc, A, st, d_err);
        uint32_t* head = A.alloc<uint32_t>(nc);
        uint64_t* hpos = A.alloc<uint64_t>(nc + 1);
        k_run_heads<<<grid(nc, 256), 256, 0, st>>>(nc, skey, head);
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(head, hpos, nc, A, st, hpos + nc);
        const uint64_t nruns = read_dev(hpos + nc, st);
        uint64_t* run_start = A.alloc<uint64_t>(nruns + 1);
        k_run_starts<<<grid(nc, 256), 256, 0, st>>>(nc, head, hpos, run_start);
        CDBG_CHECK_LAUNCH();
        uint32_t* rep = A.alloc<uint32_t>(nc);
        uint32_t* rep_first = A.alloc<uint32_t>(nc);
        uint32_t* collided = A.alloc<uint32_t>(nruns + 1);
        CDBG_CUDA(cudaMemsetAsync(rep_first, 0xff, 4 * nc, st));
        CDBG_CUDA(cudaMemsetAsync(collided, 0, 4 * (nruns + 1), st));
        {
            CDBG_PROF("k_member_match", st);
            k_member_match_raw<<<grid(nc, 256), 256, 0, st>>>(nc, head, hpos, run_start, sidx, cv, L, rep, rep_first,
                                                               collided);
        }
        CDBG_CHECK_LAUNCH();
        {
            unsigned long long* ncol = A.alloc<unsigned long long>(1);
            CDBG_CUDA(cudaMemsetAsync(ncol, 0, 8, st));
            k_count_flags<<<grid(nruns, 256), 256, 0, st>>>(nruns, collided, ncol);
            CDBG_CHECK_LAUNCH();
            if (read_dev(ncol, st)) {
                k_group_collided_raw<<<grid(nruns, 128), 128, 0, st>>>(nruns, collided, run_start, nc, sidx, cv, L,
                                                                       rep, rep_first);
                CDBG_CHECK_LAUNCH();
            }
        }
        // 2. representatives: compact, encode, look up in the dictionary
        uint32_t* is_rep = A.alloc<uint32_t>(nc);
        uint64_t* rpos = A.alloc<uint64_t>(nc + 1);
        k_rep_flags<<<grid(nc, 256), 256, 0, st>>>(nc, rep, is_rep);
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(is_rep, rpos, nc, A, st, rpos + nc);
        const uint64_t nr = read_dev(rpos + nc, st);
        cand_view rv;
        rv.kind_id = A.alloc<uint32_t>(nr + 1);
        rv.first = A.alloc<uint32_t>(nr + 1);
        rv.hash = A.alloc<uint64_t>(nr + 1);
        uint32_t* rep_index = A.alloc<uint32_t>(nc);
        k_rep_compact<<<grid(nc, 256), 256, 0, st>>>(nc, is_rep, rpos, cv, rep_first, rv, rep_index);
        CDBG_CHECK_LAUNCH();
        const uint32_t nw = (C + 31) / 32;
        int wpb = (int)std::max<uint64_t>(1, std::min<uint64_t>(8, (96 * 1024) / (4ull * nw)));
        const size_t shm = (size_t)wpb * nw * 4;
        if (shm > 48 * 1024) {
            CDBG_CUDA(cudaFuncSetAttribute(k_encode<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
            CDBG_CUDA(cudaFuncSetAttribute(k_encode<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        }
        uint64_t* cbits = A.alloc<uint64_t>(nr);
        uint64_t* cb = A.alloc<uint64_t>(nr + 1);
        {
            CDBG_PROF("k_encode", st);
            k_encode<false><<<grid(ceil_div(nr, 32), wpb), wpb * 32, shm, st>>>(nr, rv, L, C, cbits, nullptr, nullptr);
        }
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint64_t, uint64_t>(cbits, cb, nr, A, st, cb + nr);
        const uint64_t ctot = read_dev(cb + nr, st);
        const uint64_t cwn = ctot / 64 + 4;
        uint64_t* cw = A.alloc<uint64_t>(cwn);
        CDBG_CUDA(cudaMemsetAsync(cw, 0, 8 * cwn, st));
        {
            CDBG_PROF("k_encode", st);
            k_encode<true><<<grid(ceil_div(nr, 32), wpb), wpb * 32, shm, st>>>(nr, rv, L, C, nullptr, cb, cw);
        }
        CDBG_CHECK_LAUNCH();
        uint32_t* rcid = A.alloc<uint32_t>(nr + 1);
        {
            CDBG_PROF("k_dict_lookup", st);
            k_dict_lookup<<<grid(nr, 256), 256, 0, st>>>(nr, rv, cw, cb, dict.view(), rcid);
        }
        CDBG_CHECK_LAUNCH();
        // 3. new classes in order of first appearance
        uint32_t* nflag = A.alloc<uint32_t>(nr);
        uint64_t* npos = A.alloc<uint64_t>(nr + 1);
        k_new_flags<<<grid(nr, 256), 256, 0, st>>>(nr, rcid, nflag);
        CDBG_CHECK_LAUNCH();
        prim::exclusive_scan<uint32_t, uint64_t>(nflag, npos, nr, A, st, npos + nr);
        const uint64_t nnew = read_dev(npos + nr, st);
        if (nnew) {
            uint64_t* rkey = A.alloc<uint64_t>(nnew);
            uint32_t* rcand = A.alloc<uint32_t>(nnew);
            k_new_reps<<<grid(nr, 256), 256, 0, st>>>(nr, rcid, npos, rv, rkey, rcand);
            CDBG_CHECK_LAUNCH();
            prim::radix_sort_pairs<uint32_t>(rkey, rcand, nnew, 0, 32, A, st, d_err);
            const uint64_t base = dict.n;
            k_assign_new<<<grid(nnew, 256), 256, 0, st>>>(nnew, rcand, base, rcid);
            CDBG_CHECK_LAUNCH();
            uint64_t* nbits = A.alloc<uint64_t>(nnew);
            uint64_t* nh = A.alloc<uint64_t>(nnew);
            uint64_t* boff = A.alloc<uint64_t>(nnew + 1);
            unsigned long long* ints = A.alloc<unsigned long long>(1);
            CDBG_CUDA(cudaMemsetAsync(ints, 0, 8, st));
            k_new_sizes<<<grid(nnew, 256), 256, 0, st>>>(nnew, rcand, rv, L, cb, nbits, nh, ints);
            CDBG_CHECK_LAUNCH();
            prim::exclusive_scan<uint64_t, uint64_t>(nbits, boff, nnew, A, st, boff + nnew);
            const uint64_t badd = read_dev(boff + nnew, st);
            add_offsets(boff, nnew + 1, dict.nbits, boff, st);  // absolute bit offsets
            if (p.copy_st && (dict.bit_off.cap < base + nnew + 1 ||
                              dict.words.cap < (dict.nbits + badd + 63) / 64 + 4)) {
                // growing frees the old arrays: after the host copies that read them
                CDBG_CUDA(cudaEventRecord(p.copy_ev, p.copy_st));
                CDBG_CUDA(cudaStreamWaitEvent(st, p.copy_ev, 0));
            }
            dict.cls_hash.reserve(base + nnew, st);
            dict.bit_off.reserve(base + nnew + 1, st);
            CDBG_CUDA(cudaMemcpyAsync(dict.cls_hash.p + base, nh, 8 * nnew, cudaMemcpyDeviceToDevice, st));
            CDBG_CUDA(cudaMemcpyAsync(dict.bit_off.p + base, boff, 8 * (nnew + 1), cudaMemcpyDeviceToDevice, st));
            dict.words.reserve((dict.nbits + badd + 63) / 64 + 4, st, true);
            {
                CDBG_PROF("k_append_bits", st);
                k_append_bits<<<grid(nnew, 8), 256, 0, st>>>(nnew, rcand, cw, cb, boff, dict.words.p);
            }
            CDBG_CHECK_LAUNCH();
            dict.total_integers += read_dev(ints, st);
            dict.n = base + nnew;
            dict.cls_hash.n = dict.n;
            dict.bit_off.n = dict.n + 1;
            dict.nbits += badd;
            dict.words.n = (dict.nbits + 63) / 64;
            dict.ensure_table(base, st, d_err);
        }
        // 4. every candidate takes its representative's class id
        k_cand_cid<<<grid(nc, 256), 256, 0, st>>>(nc, rep, rep_index, rcid, cid);
        CDBG_CHECK_LAUNCH();
    }
    // ---- node class ids
    uint32_t* n_cid = A.alloc<uint32_t>(D);
    {
        CDBG_PROF("k_node_cid", st);
        k_node_cid<<<grid(D, 256), 256, 0, st>>>(D, n_rec, (uint32_t)R0, rec_cand, nrc, mgrp, cid, n_cid);
    }
    CDBG_CHECK_LAUNCH();
    // ---- chains (extension masks and links were made with the tables)
    chain_ws W;
    W.link = link;
    W.meta = n_meta;
    W.mask = n_mask;
    W.ch_node = A.alloc<uint32_t>(D);
    W.ch_rc = A.alloc<uint8_t>(D);
    W.ch_ord = A.alloc<unsigned long long>(D);
    W.ch_vis = A.alloc<uint8_t>(D);
    W.fe = A.alloc<uint32_t>(D);
    W.seed_start = A.alloc<uint32_t>(D);
    W.seed_len = A.alloc<uint32_t>(D);
    W.seed_open = A.alloc<uint8_t>(D);
    W.covered = A.alloc<uint8_t>(D);
    W.cursor = A.alloc<unsigned long long>(1);
    W.D = D;
    CDBG_CUDA(cudaMemsetAsync(W.seed_len, 0, 4 * D, st));
    CDBG_CUDA(cudaMemsetAsync(W.covered, 0, D, st));
    CDBG_CUDA(cudaMemsetAsync(W.cursor, 0, 8, st));
    {
        uint32_t* ends = A.alloc<uint32_t>(D);
        unsigned long long* cnt2 = A.alloc<unsigned long long>(2);
        CDBG_CUDA(cudaMemsetAsync(cnt2, 0, 16, st));
        {
            CDBG_PROF("k_chain_ends", st);
            k_chain_ends<<<grid(D, 256), 256, 0, st>>>(W, ends, cnt2);
        }
        CDBG_CHECK_LAUNCH();
        const uint64_t nends = read_dev(cnt2, st);
        uint4* heads = A.alloc<uint4>(nends + 1);
        if (nends) {
            CDBG_PROF("k_chain_lead", st);
            k_chain_lead<<<grid(nends, 256), 256, 0, st>>>(W, ends, nends, heads, cnt2 + 1, d_err);
        }
        CDBG_CHECK_LAUNCH();
        const uint64_t nheads = read_dev(cnt2 + 1, st);
        if (nheads) {
            CDBG_PROF("k_chain_paths", st);
            k_chain_paths<<<grid(nheads, 128), 128, 0, st>>>(W, heads, nheads);
        }
        CDBG_CHECK_LAUNCH();
    }
    {
        CDBG_PROF("k_chain_cycles", st);
        k_chain_cycles<<<grid(D, 128), 128, 0, st>>>(W, d_err);
    }
    CDBG_CHECK_LAUNCH();
    // ---- fragments, in seed order
    uint32_t* is_seed = A.alloc<uint32_t>(D);
    uint64_t* fpos = A.alloc<uint64_t>(D + 1);
    k_seed_flags<<<grid(D, 256), 256, 0, st>>>(D, W.seed_len, is_seed);
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint32_t, uint64_t>(is_seed, fpos, D, A, st, fpos + D);
    const uint64_t nfr = read_dev(fpos + D, st);
    check_device_error_word(d_err, st, "unitig walk");
    uint32_t* seed_of = A.alloc<uint32_t>(nfr + 1);
    k_seed_list<<<grid(D, 256), 256, 0, st>>>(D, is_seed, fpos, seed_of);
    CDBG_CHECK_LAUNCH();
    uint64_t* fsz = A.alloc<uint64_t>(nfr + 1);
    uint64_t* foff = A.alloc<uint64_t>(nfr + 1);
    unsigned long long* seqt = A.alloc<unsigned long long>(1);
    CDBG_CUDA(cudaMemsetAsync(seqt, 0, 8, st));
    if (nfr) {
        CDBG_PROF("k_frag_sizes", st);
        k_frag_sizes<<<grid(nfr, 256), 256, 0, st>>>(nfr, seed_of, W.seed_start, W.seed_len, W.fe, n_cid, k, fsz, seqt);
    }
    CDBG_CHECK_LAUNCH();
    prim::exclusive_scan<uint64_t, uint64_t>(fsz, foff, nfr, A, st, foff + nfr);
    const uint64_t fbytes = read_dev(foff + nfr, st);
    uint8_t* fb = A.alloc<uint8_t>(fbytes + 8);
    if (nfr) {
        CDBG_PROF("k_frag_write", st);
        k_frag_write<K><<<grid(nfr, FW_THREADS), FW_THREADS, 0, st>>>(nfr, seed_of, W.seed_start, W.seed_len,
                                                                       W.seed_open, W.fe, n_cid, n_key, k, foff, fb);
    }
    CDBG_CHECK_LAUNCH();
    const uint64_t seq_total = read_dev(seqt, st);
    out.n_fragments += nfr;
    out.total_seq_bytes += seq_total;
    out.n_occ += nocc;
    out.n_distinct += D;
    if (p.to_host) {
        const size_t o = out.frag.size();
        out.frag.resize(o + fbytes);
        CDBG_CUDA(cudaMemcpyAsync(out.frag.data() + o, fb, fbytes, cudaMemcpyDeviceToHost, st));
    } else {
        const uint64_t old_n = dfrag.n;
        if (p.copy_st && dfrag.n + fbytes + 8 > dfrag.cap) {
            // growing frees the old buffer: after the host copies that read it
            CDBG_CUDA(cudaEventRecord(p.copy_ev, p.copy_st));
            CDBG_CUDA(cudaStreamWaitEvent(st, p.copy_ev, 0));
        }
        dfrag.reserve(dfrag.n + fbytes + 8, st);
        CDBG_CUDA(cudaMemcpyAsync(dfrag.p + dfrag.n, fb, fbytes, cudaMemcpyDeviceToDevice, st));
        dfrag.n += fbytes;
        if (p.keep_frag_offsets && nfr) {
            dfoff.reserve(dfoff.n + nfr + 1, st);
            add_offsets(foff, nfr, old_n, dfoff.p + dfoff.n, st);
            dfoff.n += nfr;
        }
        if (p.copy_st && p.frag_host && out.frag_host_copied == old_n && dfrag.n <= p.frag_host_cap && fbytes) {
            // this batch's fragments go to the host while the next batch runs
            CDBG_CUDA(cudaEventRecord(p.copy_ev, st));
            CDBG_CUDA(cudaStreamWaitEvent(p.copy_st, p.copy_ev, 0));
            CDBG_CUDA(cudaMemcpyAsync(p.frag_host + old_n, dfrag.p + old_n, fbytes, cudaMemcpyDeviceToHost,
                                      p.copy_st));
            out.frag_host_copied = dfrag.n;
            if (p.on_frag) p.on_frag(p.on_frag_ctx, old_n, fbytes);
        }
    }
    if (!p.to_host && p.copy_st) {
        // completed class words (all but the one later classes still fill) and
        // class offsets go to the host while the next batch runs
        const uint64_t wdone = dict.nbits / 64;
        const bool words_go = p.words_host && out.words_host_copied < wdone && wdone <= p.words_host_cap;
        const bool offs_go = p.offs_host && out.offs_host_copied < dict.n && dict.n <= p.offs_host_cap;
        if (words_go || offs_go) {
            CDBG_CUDA(cudaEventRecord(p.copy_ev, st));
            CDBG_CUDA(cudaStreamWaitEvent(p.copy_st, p.copy_ev, 0));
        }
        if (words_go) {
            CDBG_CUDA(cudaMemcpyAsync(p.words_host + out.words_host_copied, dict.words.p + out.words_host_copied,
                                      8 * (wdone - out.words_host_copied), cudaMemcpyDeviceToHost, p.copy_st));
            out.words_host_copied = wdone;
        }
        if (offs_go) {
            CDBG_CUDA(cudaMemcpyAsync(p.offs_host + out.offs_host_copied, dict.bit_off.p + out.offs_host_copied,
                                      8 * (dict.n - out.offs_host_copied), cudaMemcpyDeviceToHost, p.copy_st));
            out.offs_host_copied = dict.n;
        }
    }
    CDBG_CUDA(cudaStreamSynchronize(st));
    out.frag_nbytes += fbytes;
    check_device_error_word(d_err, st, "phase-2 batch");
    A.release(mark);
}

}  // namespace
}  // namespace cdbg

namespace cdbg {

namespace {
template <typename K>
void run_all(record_set const& rs, phase2_params const& p, dev_arena& A, cudaStream_t st, uint32_t* d_err,
             phase2_result& out) {
    const uint64_t n = rs.n;
    const uint32_t B = rs.B;
    auto mark = A.mark();
    uint64_t* nk = A.alloc<uint64_t>(n + 1);
    uint32_t* rbucket = A.alloc<uint32_t>(n + 1);
    uint64_t* rhash = A.alloc<uint64_t>(n + 1);
    uint64_t* occ = A.alloc<uint64_t>(n + 1);
    if (n) {
        {
            CDBG_PROF("k_rec_prep", st);
            k_rec_prep<<<grid(n, 256), 256, 0, st>>>(n, rs.len, p.k, rs.bucket_start, B, nk, rbucket, rs.col_off,
                                                     rs.colors, rhash);
        }
        CDBG_CHECK_LAUNCH();
    }
    prim::exclusive_scan<uint64_t, uint64_t>(nk, occ, n, A, st, occ + n);
    uint64_t* d_bocc = A.alloc<uint64_t>(B + 1);
    k_gather_u64<<<grid(B + 1, 256), 256, 0, st>>>(B + 1, occ, rs.bucket_start, d_bocc);
    CDBG_CHECK_LAUNCH();
    std::vector<uint64_t> bocc(B + 1), hbstart(B + 1);
    read_small(bocc.data(), d_bocc, 8ull * (B + 1), st);
    read_small(hbstart.data(), rs.bucket_start, 8ull * (B + 1), st);
    uint64_t budget = p.batch_occ;
    if (budget == 0) {
        int dev = 0;
        CDBG_CUDA(cudaGetDevice(&dev));
        const uint64_t avail = std::min<uint64_t>(device_available(dev) + A.cached_free(), A.headroom());
        // ~200 B of device memory per k-mer occurrence in the batch, worst
        // case; keep 45% of the available memory for outputs and the dictionary
        budget = std::max<uint64_t>(1ull << 22, std::min<uint64_t>(1ull << 28, (uint64_t)(avail * 0.5) / 220));
    }
    rec_view R{rs.start, rs.len, rs.flags, rs.col_off, rs.colors, rbucket, occ, rs.words};
    phase2_state local_state;
    phase2_state& S = out.state ? *out.state : local_state;
    class_dict dict(S);
    if (p.keep_dict) {
        dict.n = S.n;
        dict.nbits = S.nbits;
        dict.total_integers = S.total_integers;
        dict.mask = S.mask;
    } else {
        dict.init(st);
    }
    dvec<uint8_t>& dfrag = S.frag;
    dfrag.n = 0;
    S.frag_off.n = 0;
    uint32_t b = 0;
    while (b < B) {
        const uint32_t s = b;
        uint64_t acc = 0, recs = 0;
        while (b < B) {
            const uint64_t ob = bocc[b + 1] - bocc[b];
            const uint64_t rb = hbstart[b + 1] - hbstart[b];
            if (b > s && (acc + ob > budget || recs + rb > MAX_BATCH_RECORDS)) break;
            acc += ob;
            recs += rb;
            ++b;
        }
        run_batch<K>(rs, R, p, s, b, bocc, A, st, d_err, dict, out, hbstart, rhash, dfrag, S.frag_off);
    }
    // outputs
    S.n = dict.n;
    S.nbits = dict.nbits;
    S.total_integers = dict.total_integers;
    S.mask = dict.mask;
    out.n_classes = dict.n;
    out.nbits = dict.nbits;
    out.total_integers = dict.total_integers;
    const uint64_t nwords = (dict.nbits + 63) / 64;
    if (p.to_host && p.copy_dict) {
        out.words.resize(nwords);
        out.offsets.resize(dict.n);
        if (nwords)
            CDBG_CUDA(cudaMemcpyAsync(out.words.data(), dict.words.p, 8 * nwords, cudaMemcpyDeviceToHost, st));
        if (dict.n)
            CDBG_CUDA(cudaMemcpyAsync(out.offsets.data(), dict.bit_off.p, 8 * dict.n, cudaMemcpyDeviceToHost, st));
    }
    CDBG_CUDA(cudaStreamSynchronize(st));
    A.release(mark);
    if (!p.to_host) {
        // outputs stay in the persistent state
        out.d_frag = S.frag.p;
        out.d_words = S.words.p;
        out.d_offsets = S.bit_off.p;
    }
}
}  // namespace

void run_phase2(record_set const& rs, phase2_params const& p, dev_arena& A, cudaStream_t st, uint32_t* d_err,
                phase2_result& out) {
    {
        // keep the caller's persistent storage across the reset
        phase2_state* S = out.state;
        out = phase2_result();
        out.state = S;
    }
    if (!p.to_host && !out.state) throw std::runtime_error("device-resident phase-2 outputs need persistent storage");
    if (p.k < 2 || p.k > 63) throw std::runtime_error("k must be in [2, 63]");
    if (p.num_colors == 0) throw std::runtime_error("num_colors must be > 0");
    if (rs.n >= (1ull << 31)) throw std::runtime_error("more than 2^31 bucket records in one build");
    phase2_params q = p;
    // bitmaps cost C/8 bytes per multi-record k-mer: lists above 8192 colors
    if (q.num_colors > 8192) q.union_bitmaps = false;
    if (q.k <= 31)
        run_all<uint64_t>(rs, q, A, st, d_err, out);
    else
        run_all<u128>(rs, q, A, st, d_err, out);
}

namespace {
// One value per thread: its l low bits OR-ed into the low vector (a value
// spans at most two words) and its bit in the high vector.
__global__ void k_ef_encode(uint64_t const* __restrict__ offsets, uint64_t nclasses, uint64_t total, uint64_t l,
                            unsigned long long* __restrict__ low, unsigned long long* __restrict__ high) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nclasses) return;
    const uint64_t v = i < nclasses ? offsets[i] : total;
    if (l) {
        const uint64_t pos = i * l, lo = v & ((uint64_t(1) << l) - 1);
        atomicOr(&low[pos >> 6], (unsigned long long)(lo << (pos & 63)));
        if ((pos & 63) + l > 64) atomicOr(&low[(pos >> 6) + 1], (unsigned long long)(lo >> (64 - (pos & 63))));
    }
    const uint64_t hp = (v >> l) + i;
    atomicOr(&high[hp >> 6], 1ull << (hp & 63));
}
}  // namespace

void ef_encode(uint64_t const* d_offsets, uint64_t nclasses, uint64_t total_bits, dev_arena& A, cudaStream_t st,
               ef_encoded& out) {
    out = ef_encoded();
    const uint64_t n = nclasses + 1, U = total_bits;
    uint64_t l = 0;
    if (U > n) {
        const uint64_t q = U / n;
        while ((uint64_t(1) << (l + 1)) <= q) ++l;
    }
    out.n = n;
    out.l = l;
    out.high_bits = n + (U >> l) + 1;
    out.low_words = (n * l + 63) / 64;
    out.high_words = (out.high_bits + 63) / 64;
    out.low = A.alloc<uint64_t>(out.low_words + 1);
    out.high = A.alloc<uint64_t>(out.high_words + 1);
    CDBG_CUDA(cudaMemsetAsync(out.low, 0, 8 * (out.low_words + 1), st));
    CDBG_CUDA(cudaMemsetAsync(out.high, 0, 8 * (out.high_words + 1), st));
    {
        CDBG_PROF("k_ef_encode", st);
        k_ef_encode<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_offsets, nclasses, U, l,
                                                                  (unsigned long long*)out.low,
                                                                  (unsigned long long*)out.high);
    }
    CDBG_CHECK_LAUNCH();
}

}  // namespace cdbg
