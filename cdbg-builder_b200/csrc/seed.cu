// Round 0 of the phase-3 stitch (the frag-file seed) on sm_100a.
//
// Restates phase3_stitch/stitch_extmem.hpp:930-944 (ext_seed_one) over all
// fragments at once.  Per fragment (frag_unitigs.bin record, unitig_spill.hpp:
// 491-522: [u8 open_flags][u32 nruns][nruns x (u64 cid, u32 num_kmers)]
// [u32 seq_len][seq_len ASCII bases]):
//
//  info    one thread: the tig's random state, FNV-1a over the ASCII bases
//          (ext_seed_from_seq, :244-251).  A closed fragment (open_flags 0)
//          is split at its color runs (ext_split_monochromatic, :113-150):
//          extremal COLOR_RUN_FOREIGN runs dropped, interior ones skipped,
//          one unitig per remaining run.  An open one presents a side
//          (ext_choose_side, :287-304: the splitmix64 finalizer's top bit of
//          the state when both ends are open), whose canonical boundary k-mer
//          (side_kmer_canonical, :261-274) is hashed to its round-store bucket
//          ((kmer_hasher(x) >> 1) % buckets, ext_route :609-620).
//  order   a stable radix sort of the fragments by bucket: within a bucket the
//          tigs keep fragment order, which is the order a one-thread seed
//          appends them to the bucket's round file.  The sizes scanned in that
//          order give each tig's position, scattered back to its fragment.
//  write   in fragment order (the records are read as they lie), one warp per
//          32 fragments writes each tig at its position in the round store's
//          layout (ext_tig_serialize, :407-428: [u8 open_flags][u64 rng]
//          [u32 nruns][runs][u32 seq_len][2-bit bases, base i at bits 2(i%4)
//          of byte i/4]) and each closed fragment's unitigs as frag records.
//
// The bytes of a fragment are read twice (info, write), in order both times;
// only the per-fragment sizes and positions move in bucket order.

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <stdexcept>
#include <string>

#include "device_kmer.cuh"
#include "primitives.cuh"
#include "seed.cuh"

namespace cdbg {
namespace {

constexpr uint64_t FNV_OFFSET = 1469598103934665603ull;  // FNV-1a 64-bit offset basis
constexpr uint64_t FNV_PRIME = 1099511628211ull;         // FNV-1a 64-bit prime
constexpr uint64_t COLOR_FOREIGN = ~0ull;                 // COLOR_RUN_FOREIGN (bucket_walker.hpp:96)
constexpr uint8_t OPEN_LEFT = 1, OPEN_RIGHT = 2;          // UNITIG_OPEN_* (bucket_walker.hpp:80-81)
constexpr uint32_t TIG_HEAD = 13;                         // u8 flags + u64 rng + u32 nruns
constexpr uint32_t PIECE_HEAD = 21;                       // u8 flags + u32 1 + u64 cid + u32 m + u32 len

inline unsigned grid(uint64_t n, unsigned t) { return (unsigned)ceil_div(n, t); }

__device__ __forceinline__ uint32_t ld_u32(uint8_t const* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
__device__ __forceinline__ uint64_t ld_u64(uint8_t const* p) { return (uint64_t)ld_u32(p) | ((uint64_t)ld_u32(p + 4) << 32); }
__device__ __forceinline__ uint64_t min64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// nuc_to_2bit (kmer.hpp:35-52): A/C/G/T (either case) -> 0..3, else 0xff.
__device__ __forceinline__ uint32_t base_code(uint32_t c) {
    switch (c | 0x20) {
        case 'a': return 0;
        case 'c': return 1;
        case 'g': return 2;
        case 't': return 3;
        default: return 0xff;
    }
}

// FNV-1a step: h * FNV_PRIME with FNV_PRIME = 2^40 + 0x1b3.
static_assert(FNV_PRIME == (1ull << 40) + 0x1b3ull, "FNV-1a 64-bit prime");
__device__ __forceinline__ uint64_t fnv_step(uint64_t h, uint32_t c) {
    h ^= c;
    return h * 0x1b3ull + (h << 40);
}

// FNV-1a over F[s, s + len) from aligned 32-bit words (F is 4-byte aligned
// with at least 4 readable bytes past the end): the partial words at either
// end byte by byte, the whole words between them four bytes at a time.  A zero
// result maps to the golden-ratio constant, as ext_seed_from_seq keeps
// xorshift off its fixed point.
__device__ uint64_t fnv_range(uint8_t const* __restrict__ F, uint64_t s, uint64_t len) {
    uint64_t h = FNV_OFFSET;
    const uint64_t e = s + len;
    uint64_t w = s & ~3ull;
    if (w < s) {
        const uint32_t x = __ldg(reinterpret_cast<uint32_t const*>(F + w));
        for (uint64_t pos = s; pos < w + 4 && pos < e; ++pos) h = fnv_step(h, (x >> (8 * (pos - w))) & 0xffu);
        w += 4;
    }
    for (; w + 4 <= e; w += 4) {
        const uint32_t x = __ldg(reinterpret_cast<uint32_t const*>(F + w));
        h = fnv_step(h, x & 0xffu);
        h = fnv_step(h, (x >> 8) & 0xffu);
        h = fnv_step(h, (x >> 16) & 0xffu);
        h = fnv_step(h, x >> 24);
    }
    if (w < e) {
        const uint32_t x = __ldg(reinterpret_cast<uint32_t const*>(F + w));
        for (uint64_t pos = w; pos < e; ++pos) h = fnv_step(h, (x >> (8 * (pos - w))) & 0xffu);
    }
    return h ? h : 0x9e3779b97f4a7c15ull;
}

struct rec_view {
    uint64_t p;       // record start
    uint8_t of;       // open flags
    uint32_t nruns;
    uint64_t runs;    // byte offset of the first run
    uint32_t len;     // bases
    uint64_t s;       // byte offset of the first base
};

__device__ __forceinline__ bool view_record(uint8_t const* __restrict__ F, uint64_t p, uint64_t q, rec_view& v) {
    if (q < p + 9) return false;
    v.p = p;
    v.of = F[p];
    v.nruns = ld_u32(F + p + 1);
    v.runs = p + 5;
    const uint64_t lp = v.runs + 12ull * v.nruns;
    if (lp + 4 > q) return false;
    v.len = ld_u32(F + lp);
    v.s = lp + 4;
    return v.s + v.len == q;
}

// Unitigs a closed fragment splits into: [lo, hi) after the extremal foreign
// runs, the k-mer offset of run lo, and (when count) their number and bytes.
__device__ __forceinline__ void closed_span(uint8_t const* __restrict__ F, rec_view const& v, uint32_t& lo,
                                            uint32_t& hi, uint64_t& base) {
    lo = 0;
    hi = v.nruns;
    if (lo < hi && ld_u64(F + v.runs) == COLOR_FOREIGN) ++lo;
    if (lo < hi && ld_u64(F + v.runs + 12ull * (hi - 1)) == COLOR_FOREIGN) --hi;
    base = lo ? ld_u32(F + v.runs + 8) : 0;
}

template <typename K>
__global__ void k_seed_info(uint8_t const* __restrict__ F, uint64_t const* __restrict__ off, uint64_t n, uint32_t k,
                            uint32_t nb, uint32_t* __restrict__ key, uint32_t* __restrict__ idx,
                            uint64_t* __restrict__ rng, uint64_t* __restrict__ tsz, uint64_t* __restrict__ csz,
                            unsigned long long* __restrict__ counts, uint32_t* err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool routed = false, closed = false;
    uint32_t pieces = 0;
    uint64_t rbytes = 0;
    if (i < n) {
        idx[i] = (uint32_t)i;
        key[i] = nb;
        tsz[i] = 0;
        csz[i] = 0;
        rec_view v;
        if (!view_record(F, off[i], off[i + 1], v)) {
            set_error(err, ERR_BAD_RECORD);
        } else {
            const uint64_t h = fnv_range(F, v.s, v.len);
            rng[i] = h;
            if (k < 2 || v.of == 0) {
                closed = true;
                uint32_t lo, hi;
                uint64_t base;
                closed_span(F, v, lo, hi, base);
                uint64_t bytes = 0;
                bool bad = false;
                for (uint32_t r = lo; r < hi; ++r) {
                    const uint64_t ro = v.runs + 12ull * r;
                    const uint32_t m = ld_u32(F + ro + 8);
                    if (ld_u64(F + ro) != COLOR_FOREIGN) {
                        // std::string::substr: throws past the end, clamps the length
                        if (base > v.len) bad = true;
                        const uint64_t want = (uint64_t)m + k - 1, room = v.len - min64(base, v.len);
                        bytes += PIECE_HEAD + min64(want, room);
                        ++pieces;
                    }
                    base += m;
                }
                if (bad) set_error(err, ERR_BAD_RECORD);
                csz[i] = bytes;
            } else {
                const bool l = v.of & OPEN_LEFT, rt = v.of & OPEN_RIGHT;
                const bool right = (l && rt) ? (mix64(h) >> 63) != 0 : !l;
                if (v.len < k) {
                    set_error(err, ERR_BAD_RECORD);
                } else {
                    const uint64_t b0 = right ? v.s + v.len - k : v.s;
                    K fwd = 0;
                    bool ok = true;
                    for (uint32_t t = 0; t < k; ++t) {
                        const uint32_t c = base_code(F[b0 + t]);
                        ok &= c < 4;
                        fwd = (fwd << 2) | (K)(c & 3);
                    }
                    if (!ok) set_error(err, ERR_BAD_RECORD);
                    const K rc = kmer_ops<K>::revcomp(fwd, k);
                    const K canon = fwd <= rc ? fwd : rc;
                    key[i] = (uint32_t)((kmer_ops<K>::hash(canon) >> 1) % nb);
                    tsz[i] = TIG_HEAD + 12ull * v.nruns + 4 + ((uint64_t)v.len + 3) / 4;
                    routed = true;
                    rbytes = off[i + 1] - off[i];
                }
            }
        }
    }
    // warp-aggregated counters: routed, closed fragments, unitigs
    const uint32_t br = __ballot_sync(0xffffffffu, routed), bc = __ballot_sync(0xffffffffu, closed);
    uint32_t pc = pieces;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        pc += __shfl_xor_sync(0xffffffffu, pc, o);
        rbytes += __shfl_xor_sync(0xffffffffu, rbytes, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (br) atomicAdd(counts + 0, (unsigned long long)__popc(br));
        if (bc) atomicAdd(counts + 1, (unsigned long long)__popc(bc));
        if (pc) atomicAdd(counts + 2, (unsigned long long)pc);
        if (rbytes) atomicAdd(counts + 3, (unsigned long long)rbytes);
    }
}

// Tig sizes in bucket order.
__global__ void k_seed_gather_sizes(uint32_t const* __restrict__ idx, uint64_t const* __restrict__ tsz, uint64_t m,
                                    uint64_t* __restrict__ out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) out[j] = tsz[idx[j]];
}

// bucket_off[b] = byte offset of bucket b's first tig: tig j starts the
// buckets (key[j - 1], key[j]].  Entry m (key nb) closes the list.
__global__ void k_seed_bucket_bounds(uint32_t const* __restrict__ key, uint64_t m, uint32_t nb,
                                     uint64_t const* __restrict__ toff, uint64_t* __restrict__ bucket_off) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j > m) return;
    const uint32_t kj = j < m ? key[j] : nb;
    const int64_t kp = j == 0 ? -1 : (int64_t)key[j - 1];
    for (int64_t b = kp + 1; b <= (int64_t)kj; ++b) bucket_off[b] = toff[j];
}

// dst[i] = byte offset of fragment i's tig: the inverse of the bucket order.
__global__ void k_seed_scatter_dst(uint32_t const* __restrict__ idx, uint64_t const* __restrict__ toff, uint64_t m,
                                   uint64_t* __restrict__ dst) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) dst[idx[j]] = toff[j];
}

// The write pass, in fragment order: one warp per 32 consecutive fragments,
// whose records are contiguous in F.  Each lane loads one fragment's offsets;
// then the warp's four groups of 8 lanes take the fragments four at a time,
// a group on the bytes of one: an open fragment's tig at its bucket position
// (ext_tig_serialize layout: [u8 flags][u64 rng] then the record's
// [u32 nruns][runs][u32 seq_len] as they are, then bases 4q..4q+3 in byte q,
// nuc_to_2bit(c) << 2(i%4) OR-ed), a closed one's unitigs as frag records
// ([flags][u32 1][u64 cid][u32 m][u32 len][bases]) at its place in the closed
// stream.
constexpr uint32_t WG = 8;  // lanes per fragment

// nuc_to_2bit of one byte without a table: (c >> 1) & 3 is A0 C1 T2 G3 for
// either case, and bit 2 of c swaps G and T; any other byte gives 0xff.
__device__ __forceinline__ uint32_t code2(uint32_t c) {
    const uint32_t lc = c | 0x20;
    const bool ok = lc == 'a' || lc == 'c' || lc == 'g' || lc == 't';
    return ok ? (((c >> 1) & 3) ^ ((c >> 2) & 1)) : 0xffu;
}

__global__ void k_seed_write(uint8_t const* __restrict__ F, uint64_t const* __restrict__ off, uint64_t n, uint32_t k,
                             uint64_t const* __restrict__ rng, uint64_t const* __restrict__ tsz,
                             uint64_t const* __restrict__ dst, uint64_t const* __restrict__ csz,
                             uint64_t const* __restrict__ coff, uint8_t* __restrict__ T, uint8_t* __restrict__ C) {
    const uint64_t i0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) << 5;
    const uint32_t lane = threadIdx.x & 31, gl = lane % WG, grp = lane / WG;
    if (i0 >= n) return;
    const uint64_t i = i0 + lane;
    unsigned long long mp = 0, mq = 0, mh = 0, md = 0;
    uint32_t kind = 0;  // 1 tig, 2 closed unitigs
    if (i < n) {
        mp = off[i];
        mq = off[i + 1];
        if (tsz[i]) {
            kind = 1;
            mh = rng[i];
            md = dst[i];
        } else if (csz[i]) {
            kind = 2;
            md = coff[i];
        }
    }
    for (uint32_t t0 = 0; t0 < 32; t0 += 32 / WG) {
        const uint32_t t = t0 + grp;
        const uint32_t kd = __shfl_sync(0xffffffffu, kind, t);
        const uint64_t p = __shfl_sync(0xffffffffu, mp, t), q = __shfl_sync(0xffffffffu, mq, t);
        const uint64_t o = __shfl_sync(0xffffffffu, md, t), h = __shfl_sync(0xffffffffu, mh, t);
        if (!kd) continue;
        rec_view v;
        view_record(F, p, q, v);
        if (kd == 1) {
            uint8_t* __restrict__ d = T + o;
            const uint64_t head = TIG_HEAD + 12ull * v.nruns + 4;
            for (uint64_t x = gl; x < head; x += WG)
                d[x] = x == 0 ? v.of : x < 9 ? (uint8_t)(h >> (8 * (x - 1))) : F[p + 1 + (x - 9)];
            const uint64_t packed = ((uint64_t)v.len + 3) / 4;
            uint8_t const* __restrict__ sb = F + v.s;
            for (uint64_t qq = gl; qq < packed; qq += WG) {
                const uint64_t b4 = 4 * qq;
                uint32_t val = code2(sb[b4]);
                if (b4 + 1 < v.len) val |= code2(sb[b4 + 1]) << 2;
                if (b4 + 2 < v.len) val |= code2(sb[b4 + 2]) << 4;
                if (b4 + 3 < v.len) val |= code2(sb[b4 + 3]) << 6;
                d[head + qq] = (uint8_t)val;
            }
        } else {
            uint32_t lo, hi;
            uint64_t base;
            closed_span(F, v, lo, hi, base);
            uint8_t* __restrict__ d = C + o;
            for (uint32_t r = lo; r < hi; ++r) {
                const uint64_t ro = v.runs + 12ull * r;
                const uint64_t cid = ld_u64(F + ro);
                const uint32_t m = ld_u32(F + ro + 8);
                if (cid == COLOR_FOREIGN) {
                    base += m;
                    continue;
                }
                const uint64_t b0 = min64(base, v.len);
                const uint32_t plen = (uint32_t)min64((uint64_t)m + k - 1, v.len - b0);
                const uint8_t of =
                    (uint8_t)((r == lo ? (v.of & OPEN_LEFT) : 0) | (r + 1 == hi ? (v.of & OPEN_RIGHT) : 0));
                const uint64_t total = PIECE_HEAD + (uint64_t)plen;
                for (uint64_t x = gl; x < total; x += WG) {
                    uint8_t b;
                    if (x == 0)
                        b = of;
                    else if (x < 5)
                        b = x == 1 ? 1 : 0;
                    else if (x < 13)
                        b = (uint8_t)(cid >> (8 * (x - 5)));
                    else if (x < 17)
                        b = (uint8_t)(m >> (8 * (x - 13)));
                    else if (x < 21)
                        b = (uint8_t)(plen >> (8 * (x - 17)));
                    else
                        b = F[v.s + b0 + (x - PIECE_HEAD)];
                    d[x] = b;
                }
                d += total;
                base += m;
            }
        }
    }
}

void check_err(uint32_t* d_err, cudaStream_t st, char const* stage) {
    uint32_t e = 0;
    read_small(&e, d_err, 4, st);
    if (e == ERR_NONE) return;
    CDBG_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
    throw std::runtime_error(std::string("device error in ") + stage +
                             (e == ERR_BAD_RECORD ? ": malformed fragment record" : ": code " + std::to_string(e)));
}

}  // namespace

void seed_fragments(uint8_t const* F, uint64_t const* off, uint64_t n, seed_config const& c, dev_arena& A,
                    cudaStream_t st, uint32_t* d_err, seed_device_out& out) {
    if (c.num_buckets == 0) throw std::runtime_error("stitch seed: num_buckets must be > 0");
    if (c.k < 2 || c.k > (c.wide ? 64u : 32u)) throw std::runtime_error("stitch seed: k out of range for the k-mer width");
    if (n >= (1ull << 32) - 1) throw std::runtime_error("stitch seed: more than 2^32 - 2 fragments in one call");
    if (reinterpret_cast<uintptr_t>(F) & 3) throw std::runtime_error("stitch seed: fragment bytes not 4-byte aligned");
    out = seed_device_out();
    const uint32_t nb = c.num_buckets;
    out.bucket_off = A.alloc<uint64_t>(nb + 1);
    uint32_t* key = A.alloc<uint32_t>(n + 1);
    uint32_t* idx = A.alloc<uint32_t>(n + 1);
    uint64_t* rng = A.alloc<uint64_t>(n + 1);
    uint64_t* tsz = A.alloc<uint64_t>(n + 1);
    uint64_t* csz = A.alloc<uint64_t>(n + 1);
    unsigned long long* counts = A.alloc<unsigned long long>(4);
    CDBG_CUDA(cudaMemsetAsync(counts, 0, 32, st));
    if (n) {
        CDBG_PROF("k_seed_info", st);
        if (c.wide)
            k_seed_info<u128><<<grid(n, 256), 256, 0, st>>>(F, off, n, c.k, nb, key, idx, rng, tsz, csz, counts, d_err);
        else
            k_seed_info<uint64_t><<<grid(n, 256), 256, 0, st>>>(F, off, n, c.k, nb, key, idx, rng, tsz, csz, counts,
                                                                d_err);
    }
    CDBG_CHECK_LAUNCH();
    unsigned long long cnt[4];
    read_small(cnt, counts, 32, st);
    check_err(d_err, st, "stitch seed");
    out.n_routed = cnt[0];
    out.n_closed = cnt[1];
    out.n_pieces = cnt[2];
    out.routed_record_bytes = cnt[3];
    const uint64_t m = out.n_routed;
    // stable order by bucket (closed fragments carry key nb and sort last)
    int bits = 1;
    while ((1ull << bits) <= nb) ++bits;
    prim::radix_sort_pairs<uint32_t, uint32_t>(key, idx, n, 0, bits, A, st, d_err);
    uint64_t* ts = A.alloc<uint64_t>(m + 1);
    uint64_t* toff = A.alloc<uint64_t>(m + 1);
    if (m) {
        k_seed_gather_sizes<<<grid(m, 256), 256, 0, st>>>(idx, tsz, m, ts);
        CDBG_CHECK_LAUNCH();
    }
    prim::exclusive_scan<uint64_t, uint64_t>(ts, toff, m, A, st, toff + m);
    k_seed_bucket_bounds<<<grid(m + 1, 256), 256, 0, st>>>(key, m, nb, toff, out.bucket_off);
    CDBG_CHECK_LAUNCH();
    uint64_t* dst = A.alloc<uint64_t>(n + 1);
    if (m) {
        k_seed_scatter_dst<<<grid(m, 256), 256, 0, st>>>(idx, toff, m, dst);
        CDBG_CHECK_LAUNCH();
    }
    uint64_t* coff = A.alloc<uint64_t>(n + 1);
    prim::exclusive_scan<uint64_t, uint64_t>(csz, coff, n, A, st, coff + n);
    uint64_t tot[2];
    read_small(&tot[0], toff + m, 8, st);
    read_small(&tot[1], coff + n, 8, st);
    check_err(d_err, st, "stitch seed order");
    out.tig_bytes = tot[0];
    out.closed_bytes = tot[1];
    out.tigs = A.alloc<uint8_t>(out.tig_bytes + 16);
    out.closed = A.alloc<uint8_t>(out.closed_bytes + 16);
    if (n) {
        CDBG_PROF("k_seed_write", st);
        k_seed_write<<<grid(ceil_div(n, 32) * 32, 256), 256, 0, st>>>(F, off, n, c.k, rng, tsz, dst, csz, coff,
                                                                       out.tigs, out.closed);
    }
    CDBG_CHECK_LAUNCH();
}

}  // namespace cdbg
