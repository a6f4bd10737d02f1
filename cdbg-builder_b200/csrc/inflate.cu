// gzip (RFC 1952) / DEFLATE (RFC 1951) decoding on the device, one warp per
// file, and the FASTA record rules of the reference's reader (kseq, as used by
// seq_reader.hpp:66 and restated by the host reader in host/io.cpp) applied
// to the inflated bytes in place.
//
// The host reader inflates with zlib on the host threads; for collections of
// many files of a few Mbp (the pangenome shape: a file per genome) one warp
// per file on the device is several times faster, the compressed bytes are
// all that cross PCIe, and the decoded sequences are already in HBM for
// phase 1.  Everything here is a decoder written from the two RFCs; nothing
// decides a result the host reader would decide differently: streams this
// decoder does not accept go back to the host reader whole.
//
// Decoder layout (per warp): all 32 lanes run the same bit reader and table
// lookups (identical values, broadcast shared-memory reads), so control flow
// never diverges; lanes split the table construction and copies.  Output goes
// through a 4 KiB ring in shared memory, written to HBM in aligned 1 KiB
// chunks; match sources closer than the ring come from it, farther ones from
// HBM (already written).  A literal/length lookup of 11 bits yields up to
// three literals at once, or a whole match length; a distance lookup of 11
// bits a whole distance (gzip -1 writes DNA as matches of about 4 bytes at a
// few hundred bytes' distance, whose codes and extra bits fit the indexes);
// codes longer than the tables fall back to a canonical decode by length.

#include <cuda_runtime.h>
#include <stdint.h>

#include "inflate.cuh"

namespace cdbg {

namespace {

constexpr uint32_t FULL = 0xffffffffu;
constexpr int LB_LIT = 11;               // literal/length table index bits
constexpr int LB_DIST = 11;              // distance table index bits
constexpr uint32_t IF_RING = 4096;       // shared-memory output window
constexpr uint32_t IF_FLUSH = 1024;      // bytes per aligned write to HBM
constexpr int IF_WARPS = 1;              // streams per CTA
static_assert(IF_RING >= IF_FLUSH + 2 * 258, "match sources must be in the ring or already in HBM");

// RFC 1951 3.2.5: length codes 257..285 and distance codes 0..29
__constant__ uint16_t c_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                        31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t c_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                        2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t c_dist_base[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                         193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__constant__ uint8_t c_dist_extra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                         6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
// RFC 1951 3.2.7: order of the code-length code lengths
__constant__ uint8_t c_clen_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// Canonical code (RFC 1951 3.2.2) by length: codes of length l are
// first[l] .. first[l] + cnt[l] - 1, for symbols sym[base[l] ..] in order.
struct code_aux {
    uint16_t cnt[16];
    uint16_t first[16];
    uint16_t base[16];
    uint16_t sym[288];
};

struct __align__(16) warp_state {
    uint8_t ring[IF_RING];
    // literal/length lookups (LB_LIT bits of input): bits 0-4 bits consumed,
    // bits 5-7 kind: 1-3 literals (bytes at bits 8, 16, 24), K_LEN a match
    // length (bits 8-16, extra bits that fit the index already added; bits
    // 17-19 extra bits still to read), K_END end of block, K_BAD no valid
    // symbol, 0 a code longer than the index (decode by length)
    uint32_t lit[1 << LB_LIT];
    // distance lookups (LB_DIST bits): bits 0-4 bits consumed, bits 5-8
    // extra bits still to read, bits 9-24 distance (folded extra added),
    // bits 25-26 kind: 1 valid, 2 no valid distance, 0 decode by length
    uint32_t dist[1 << LB_DIST];
    uint16_t one[1 << LB_LIT];  // one symbol per lookup, (length << 9) | symbol
    code_aux la, da;
    uint32_t hist[16];
    uint8_t lens[320];
};

constexpr uint32_t K_LEN = 4, K_END = 5, K_BAD = 6;

// Little-endian bit reader over the input (RFC 1951 3.1.1: bits from the
// least significant end of each byte).  All lanes hold the same state.  The
// buffer above the `nb` valid bits holds either zeros or the input bits that
// follow (a refill ORs the next eight bytes in place, so repeated bytes land
// on identical bits); code that moves `ip` by hand clears it.
struct bit_reader {
    uint8_t const* in;  // 8-byte aligned, readable 32 bytes past `end`
    uint64_t ip;        // byte of bit `nb` of the buffer
    uint64_t end;       // end of this stream's bytes
    uint64_t bb;
    uint32_t nb;
    // afterwards at least 56 bits are buffered (bytes past `end` read as
    // whatever follows; callers check ip against end)
    __device__ __forceinline__ void refill() {
        if (nb < 56) {
            const uint64_t a = ip & ~uint64_t(7);
            const uint32_t sh = (uint32_t)(ip & 7) * 8u;
            const uint64_t w0 = __ldg(reinterpret_cast<unsigned long long const*>(in + a));
            const uint64_t w1 = __ldg(reinterpret_cast<unsigned long long const*>(in + a) + 1);
            const uint64_t v = sh ? (w0 >> sh) | (w1 << (64u - sh)) : w0;
            bb |= v << nb;
            const uint32_t take = (63u - nb) >> 3;
            ip += take;
            nb += 8u * take;
        }
    }
    __device__ __forceinline__ void drop(uint32_t n) {
        bb >>= n;
        nb -= n;
    }
    // n <= 16, at least n bits buffered
    __device__ __forceinline__ uint32_t get(uint32_t n) {
        const uint32_t v = (uint32_t)bb & ((1u << n) - 1u);
        drop(n);
        return v;
    }
    __device__ __forceinline__ bool overrun() const { return ip > end + 8; }
    // first byte not consumed (the buffer holds whole bytes after align())
    __device__ __forceinline__ uint64_t pos() const { return ip - nb / 8; }
    __device__ __forceinline__ void align() { drop(nb & 7u); }
    // continue at byte position p (nothing buffered)
    __device__ __forceinline__ void seek(uint64_t p) {
        ip = p;
        bb = 0;
        nb = 0;
    }
};

__device__ __forceinline__ uint32_t lanemask_lt_() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Decoding tables of the code with lengths lens[0, n).  Returns false for an
// over-subscribed set, and for an incomplete one unless it is a single code
// of one bit or no code at all (with `strict`, for the code-length code, any
// incomplete set) -- the sets zlib also refuses.  Warp-collective.
__device__ bool build_code(uint8_t const* lens, int n, uint16_t* tab, int lb, code_aux& a, uint32_t* hist,
                           int lane, bool strict) {
    if (lane < 16) hist[lane] = 0;
    __syncwarp();
    for (int s0 = 0; s0 < n; s0 += 32) {
        const int s = s0 + lane;
        const uint32_t l = s < n ? lens[s] : 0u;
        const uint32_t grp = __match_any_sync(FULL, l);
        if (l && lane == __ffs(grp) - 1) hist[l] += __popc(grp);
        __syncwarp();
    }
    int ok = 1;
    if (lane == 0) {
        int left = 1, maxl = 0;
        uint32_t code = 0, idx = 0, prev = 0;
        a.cnt[0] = 0;
        for (int l = 1; l < 16; ++l) {
            const uint32_t c = hist[l];
            left = 2 * left - (int)c;
            if (left < 0) ok = 0;
            code = (code + prev) << 1;
            a.cnt[l] = (uint16_t)c;
            a.first[l] = (uint16_t)code;
            a.base[l] = (uint16_t)idx;
            idx += c;
            prev = c;
            if (c) maxl = l;
        }
        if (left > 0 && (strict || maxl > 1)) ok = 0;
    }
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) return false;
    for (int i = lane; i < (1 << lb) / 2; i += 32) reinterpret_cast<uint32_t*>(tab)[i] = 0u;
    if (lane < 16) hist[lane] = 0;
    __syncwarp();
    for (int s0 = 0; s0 < n; s0 += 32) {
        const int s = s0 + lane;
        const uint32_t l = s < n ? lens[s] : 0u;
        const uint32_t grp = __match_any_sync(FULL, l);
        const uint32_t before = l ? hist[l] : 0u;
        const uint32_t rank = before + __popc(grp & lanemask_lt_());
        __syncwarp();
        if (l) {
            if (lane == __ffs(grp) - 1) hist[l] = before + __popc(grp);
            a.sym[a.base[l] + rank] = (uint16_t)s;
            if (l <= (uint32_t)lb) {
                const uint32_t rev = __brev(a.first[l] + rank) >> (32 - l);
                const uint16_t e = (uint16_t)((l << 9) | (uint32_t)s);
                for (uint32_t x = rev; x < (1u << lb); x += 1u << l) tab[x] = e;
            }
        }
        __syncwarp();
    }
    return true;
}

// Canonical decode by length (codes longer than a table's index) of the
// next bits `bb`: (bits used << 16) | symbol, or -1 for a bit string that is
// no code.
__device__ __noinline__ int decode_slow(uint64_t bb, code_aux const& a) {
    uint32_t code = 0;
    for (int len = 1; len < 16; ++len) {
        code = (code << 1) | ((uint32_t)bb & 1u);
        bb >>= 1;
        const uint32_t off = code - a.first[len];
        if (off < a.cnt[len]) return (len << 16) | a.sym[a.base[len] + off];
    }
    return -1;
}

// One symbol from a one-symbol table (at least 15 bits buffered); -1 for a
// bit string that is no code.
__device__ __forceinline__ int decode_sym(bit_reader& br, uint16_t const* tab, int lb, code_aux const& a) {
    const uint32_t e = tab[(uint32_t)br.bb & ((1u << lb) - 1u)];
    const uint32_t l = e >> 9;
    if (l) {
        br.drop(l);
        return (int)(e & 511u);
    }
    const int r = decode_slow(br.bb, a);
    if (r < 0) return -1;
    br.drop((uint32_t)r >> 16);
    return r & 0xffff;
}

// Literal/length lookups from the one-symbol table in w.one.  A literal whose
// code leaves room in the index for the next code(s), when those are
// literals too, yields two or three (the bits after a code are the index
// shifted right by its length, upper bits zero, which select the same entry
// for any code that fits); a length code whose extra bits fit in the index
// comes with them added.  Warp-collective.
__device__ void pack_litlen(warp_state& w, int lane) {
    __syncwarp();
    for (uint32_t x = (uint32_t)lane; x < (1u << LB_LIT); x += 32) {
        const uint32_t e1 = w.one[x];
        const uint32_t l1 = e1 >> 9, s1 = e1 & 511u;
        uint32_t out = 0;
        if (l1 == 0) {
            out = 0;
        } else if (s1 < 256) {
            uint32_t tot = l1, cnt = 1;
            out = s1 << 8;
            const uint32_t e2 = w.one[x >> tot];
            const uint32_t l2 = e2 >> 9, s2 = e2 & 511u;
            if (l2 && s2 < 256 && tot + l2 <= (uint32_t)LB_LIT) {
                out |= s2 << 16;
                ++cnt;
                tot += l2;
                const uint32_t e3 = w.one[x >> tot];
                const uint32_t l3 = e3 >> 9, s3 = e3 & 511u;
                if (l3 && s3 < 256 && tot + l3 <= (uint32_t)LB_LIT) {
                    out |= s3 << 24;
                    ++cnt;
                    tot += l3;
                }
            }
            out |= (cnt << 5) | tot;
        } else if (s1 == 256) {
            out = (K_END << 5) | l1;
        } else if (s1 <= 285) {
            const uint32_t i = s1 - 257, ex = c_len_extra[i];
            uint32_t len = c_len_base[i], c = l1, rem = ex;
            if (l1 + ex <= (uint32_t)LB_LIT) {
                len += (x >> l1) & ((1u << ex) - 1u);
                c = l1 + ex;
                rem = 0;
            }
            out = (rem << 17) | (len << 8) | (K_LEN << 5) | c;
        } else {
            out = (K_BAD << 5) | l1;
        }
        w.lit[x] = out;
    }
    __syncwarp();
}

// Distance lookups from the one-symbol table in w.one.  Warp-collective.
__device__ void pack_dist(warp_state& w, int lane) {
    __syncwarp();
    for (uint32_t x = (uint32_t)lane; x < (1u << LB_DIST); x += 32) {
        const uint32_t e1 = w.one[x];
        const uint32_t l1 = e1 >> 9, s1 = e1 & 511u;
        uint32_t out = 0;
        if (l1 && s1 < 30) {
            const uint32_t ex = c_dist_extra[s1];
            uint32_t d = c_dist_base[s1], c = l1, rem = ex;
            if (l1 + ex <= (uint32_t)LB_DIST) {
                d += (x >> l1) & ((1u << ex) - 1u);
                c = l1 + ex;
                rem = 0;
            }
            out = (1u << 25) | (d << 9) | (rem << 5) | c;
        } else if (l1) {
            out = (2u << 25) | l1;
        }
        w.dist[x] = out;
    }
    __syncwarp();
}

struct out_state {
    uint8_t* o;      // region in HBM
    uint32_t cap;    // (a stream of 4 GiB or more goes to the host reader)
    uint32_t op;     // bytes produced
    uint32_t fp;     // bytes written to HBM (a multiple of IF_FLUSH)
};

// Writes ring bytes [fp, fp + IF_FLUSH) to HBM (32 bytes per lane, aligned).
__device__ __forceinline__ void flush_chunk(warp_state& w, out_state& os, int lane) {
    __syncwarp();
    const uint32_t r = os.fp & (IF_RING - 1);
    uint4 const* src = reinterpret_cast<uint4 const*>(w.ring + r) + 2 * lane;
    uint4* dst = reinterpret_cast<uint4*>(os.o + os.fp) + 2 * lane;
    dst[0] = src[0];
    dst[1] = src[1];
    os.fp += IF_FLUSH;
    __syncwarp();
}

// Copies L bytes from distance d back (d <= bytes produced in this member).
// Lane i copies byte i of each 32-byte round.  Every source position lies
// before the copy (an overlapping copy, d < L, reads position op - d +
// (i mod d): the period repeats), so no lane reads what this copy writes; a
// ring slot read here is written here only when the write lands a whole ring
// later (d + L > IF_RING), and then each round's writes wait for all reads.
// The common case -- at most 32 bytes, no overlap, source in the ring -- is
// one round.
__device__ __forceinline__ void copy_match(warp_state& w, out_state& os, uint32_t d, uint32_t L, int lane) {
    __syncwarp();  // the bytes stored before are visible to every lane
    const uint32_t i = (uint32_t)lane;
    if (L <= 32 && d >= L && d + L <= IF_RING) {
        if (i < L) w.ring[(os.op + i) & (IF_RING - 1)] = w.ring[(os.op - d + i) & (IF_RING - 1)];
        os.op += L;
        return;
    }
    const bool wrap = d + L > IF_RING;
    for (uint32_t i0 = 0; i0 < L; i0 += 32) {
        const uint32_t j = i0 + i;
        uint8_t v = 0;
        if (j < L) {
            const uint32_t src = os.op - d + (d < L ? j % d : j);
            v = d <= IF_RING ? w.ring[src & (IF_RING - 1)] : os.o[src];
        }
        if (wrap) __syncwarp();
        if (j < L) w.ring[(os.op + j) & (IF_RING - 1)] = v;
    }
    os.op += L;
}

// gzip member header (RFC 1952 2.3.1) at a byte boundary.
__device__ bool read_member_header(bit_reader& br) {
    br.refill();
    if (br.get(8) != 0x1f || br.get(8) != 0x8b || br.get(8) != 8) return false;
    const uint32_t flg = br.get(8);
    if (flg & 0xe0u) return false;
    br.refill();
    br.get(16);
    br.get(16);  // MTIME
    br.refill();
    br.get(8);
    br.get(8);  // XFL, OS
    if (flg & 4u) {  // FEXTRA
        const uint32_t xlen = br.get(16);
        const uint64_t p = br.pos() + xlen;
        br.seek(p);
        if (br.overrun()) return false;
    }
    for (uint32_t bit = 8; bit <= 16; bit <<= 1) {  // FNAME, FCOMMENT: zero-terminated
        if (!(flg & bit)) continue;
        for (;;) {
            br.refill();
            if (br.overrun()) return false;
            if (br.get(8) == 0) break;
        }
    }
    if (flg & 2u) {  // FHCRC
        br.refill();
        br.get(16);
    }
    return !br.overrun();
}

__global__ void __launch_bounds__(IF_WARPS * 32) k_inflate(stream_set s) {
    __shared__ warp_state W[IF_WARPS];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t f = blockIdx.x * IF_WARPS + (uint32_t)wi;
    if (f >= s.n) return;  // whole warp
    warp_state& w = W[wi];
    const uint64_t cap64 = s.out_cap[f];
    out_state os{s.out + s.out_off[f], (uint32_t)(cap64 < 0xfffff000ull ? cap64 : 0xfffff000ull), 0, 0};
    uint32_t st = STREAM_OK;
    if (!s.gz[f]) {
        // plain file: copied as is
        const uint64_t n = s.in_len[f];
        if (n > os.cap) {
            st = STREAM_OVERFLOW;
        } else {
            uint8_t const* src = s.in + s.in_off[f];
            for (uint64_t i = (uint64_t)lane; i < n; i += 32) os.o[i] = src[i];
            os.op = (uint32_t)n;
        }
        if (lane == 0) {
            s.out_len[f] = os.op;
            s.status[f] = st;
        }
        return;
    }
    bit_reader br{s.in, s.in_off[f], s.in_off[f] + s.in_len[f], 0, 0};
    for (;;) {  // members
        if (!read_member_header(br)) {
            st = STREAM_BAD;
            break;
        }
        const uint32_t member0 = os.op;
        bool last = false;
        while (!last && st == STREAM_OK) {  // blocks
            br.refill();
            if (br.overrun()) {
                st = STREAM_BAD;
                break;
            }
            last = br.get(1) != 0;
            const uint32_t type = br.get(2);
            if (type == 0) {
                // stored: LEN, NLEN at the next byte boundary, then LEN bytes
                br.align();
                const uint32_t len = br.get(16), nlen = br.get(16);
                if ((len ^ 0xffffu) != nlen) {
                    st = STREAM_BAD;
                    break;
                }
                if ((uint64_t)os.op + len > os.cap) {
                    st = STREAM_OVERFLOW;
                    break;
                }
                const uint64_t p = br.pos();
                if (p + len > br.end) {
                    st = STREAM_BAD;
                    break;
                }
                for (uint32_t i0 = 0; i0 < len; i0 += 32) {
                    if (os.op - os.fp >= IF_FLUSH) flush_chunk(w, os, lane);
                    const uint32_t n = min(32u, len - i0);
                    if ((uint32_t)lane < n) w.ring[(os.op + lane) & (IF_RING - 1)] = br.in[p + i0 + lane];
                    os.op += n;
                    __syncwarp();
                }
                br.seek(p + len);
                continue;
            }
            if (type == 3) {
                st = STREAM_BAD;
                break;
            }
            if (type == 1) {
                // fixed codes (RFC 1951 3.2.6); 32 distance codes of 5 bits
                // (30 and 31 never valid) keep the set complete
                for (int i = lane; i < 288 + 32; i += 32)
                    w.lens[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : i < 288 ? 8 : 5;
                __syncwarp();
                build_code(w.lens, 288, w.one, LB_LIT, w.la, w.hist, lane, false);
                pack_litlen(w, lane);
                build_code(w.lens + 288, 32, w.one, LB_DIST, w.da, w.hist, lane, false);
                pack_dist(w, lane);
            } else {
                // dynamic codes (RFC 1951 3.2.7)
                const uint32_t hlit = br.get(5) + 257, hdist = br.get(5) + 1, hclen = br.get(4) + 4;
                if (hlit > 286 || hdist > 30) {
                    st = STREAM_BAD;
                    break;
                }
                for (int i = lane; i < 19; i += 32) w.lens[i] = 0;
                __syncwarp();
                for (uint32_t i = 0; i < hclen; ++i) {
                    br.refill();
                    const uint32_t v = br.get(3);
                    if (lane == 0) w.lens[c_clen_order[i]] = (uint8_t)v;
                }
                __syncwarp();
                if (!build_code(w.lens, 19, w.one, LB_LIT, w.la, w.hist, lane, true)) {
                    st = STREAM_BAD;
                    break;
                }
                const uint32_t total = hlit + hdist;
                uint32_t n = 0;
                while (n < total) {
                    br.refill();
                    if (br.overrun()) {
                        st = STREAM_BAD;
                        break;
                    }
                    const int sym = decode_sym(br, w.one, LB_LIT, w.la);
                    if (sym < 0) {
                        st = STREAM_BAD;
                        break;
                    }
                    if (sym < 16) {
                        if (lane == 0) w.lens[n] = (uint8_t)sym;
                        ++n;
                    } else {
                        uint32_t rep, val = 0;
                        if (sym == 16) {
                            if (n == 0) {
                                st = STREAM_BAD;
                                break;
                            }
                            val = w.lens[n - 1];
                            rep = 3 + br.get(2);
                        } else if (sym == 17) {
                            rep = 3 + br.get(3);
                        } else {
                            rep = 11 + br.get(7);
                        }
                        if (n + rep > total) {
                            st = STREAM_BAD;
                            break;
                        }
                        for (uint32_t j = (uint32_t)lane; j < rep; j += 32) w.lens[n + j] = (uint8_t)val;
                        n += rep;
                    }
                    __syncwarp();
                }
                if (st != STREAM_OK) break;
                __syncwarp();
                if (w.lens[256] == 0 || !build_code(w.lens, (int)hlit, w.one, LB_LIT, w.la, w.hist, lane, false)) {
                    st = STREAM_BAD;
                    break;
                }
                pack_litlen(w, lane);
                if (!build_code(w.lens + hlit, (int)hdist, w.one, LB_DIST, w.da, w.hist, lane, false)) {
                    st = STREAM_BAD;
                    break;
                }
                pack_dist(w, lane);
            }
            // the block's symbols: after a refill at least 56 bits are
            // buffered, enough for a whole match (15 + 5 + 15 + 13 bits)
            for (;;) {
                if (os.op - os.fp >= IF_FLUSH) flush_chunk(w, os, lane);
                if (br.nb < 56) {
                    br.refill();
                    if (br.overrun()) {
                        st = STREAM_BAD;
                        break;
                    }
                }
                const uint32_t e = w.lit[(uint32_t)br.bb & ((1u << LB_LIT) - 1u)];
                const uint32_t kind = (e >> 5) & 7u;
                if (kind - 1u < 3u) {  // one to three literals
                    if ((uint64_t)os.op + kind > os.cap) {
                        st = STREAM_OVERFLOW;
                        break;
                    }
                    if ((uint32_t)lane < kind) w.ring[(os.op + lane) & (IF_RING - 1)] = (uint8_t)(e >> (8 + 8 * lane));
                    os.op += kind;
                    br.drop(e & 31u);
                    continue;
                }
                uint32_t L;
                if (kind == K_LEN) {
                    br.drop(e & 31u);
                    L = ((e >> 8) & 511u) + br.get((e >> 17) & 7u);
                } else if (kind == K_END) {
                    br.drop(e & 31u);
                    break;
                } else if (kind == K_BAD) {
                    st = STREAM_BAD;
                    break;
                } else {
                    // a code longer than the index
                    const int r = decode_slow(br.bb, w.la);
                    if (r < 0) {
                        st = STREAM_BAD;
                        break;
                    }
                    br.drop((uint32_t)r >> 16);
                    const uint32_t sym = (uint32_t)r & 0xffffu;
                    if (sym < 256) {
                        if (os.op >= os.cap) {
                            st = STREAM_OVERFLOW;
                            break;
                        }
                        if (lane == 0) w.ring[os.op & (IF_RING - 1)] = (uint8_t)sym;
                        ++os.op;
                        continue;
                    }
                    if (sym == 256) break;
                    if (sym > 285) {
                        st = STREAM_BAD;
                        break;
                    }
                    L = c_len_base[sym - 257] + br.get(c_len_extra[sym - 257]);
                }
                const uint32_t de = w.dist[(uint32_t)br.bb & ((1u << LB_DIST) - 1u)];
                const uint32_t dk = de >> 25;
                uint32_t d;
                if (dk == 1) {
                    br.drop(de & 31u);
                    d = ((de >> 9) & 0xffffu) + br.get((de >> 5) & 15u);
                } else if (dk == 0) {
                    const int r = decode_slow(br.bb, w.da);
                    if (r < 0 || (r & 0xffff) >= 30) {
                        st = STREAM_BAD;
                        break;
                    }
                    br.drop((uint32_t)r >> 16);
                    const uint32_t ds = (uint32_t)r & 0xffffu;
                    d = c_dist_base[ds] + br.get(c_dist_extra[ds]);
                } else {
                    st = STREAM_BAD;
                    break;
                }
                if (d > os.op - member0) {
                    st = STREAM_BAD;
                    break;
                }
                if ((uint64_t)os.op + L > os.cap) {
                    st = STREAM_OVERFLOW;
                    break;
                }
                copy_match(w, os, d, L, lane);
            }
        }
        if (st != STREAM_OK) break;
        // trailer: CRC-32 (not checked here) and ISIZE = member size mod 2^32
        br.align();
        br.refill();
        br.get(16);
        br.get(16);
        br.refill();
        const uint32_t isize = br.get(16) | (br.get(16) << 16);
        if (br.overrun() || isize != os.op - member0) {
            st = STREAM_BAD;
            break;
        }
        const uint64_t p = br.pos();
        if (p > br.end) {
            st = STREAM_BAD;
            break;
        }
        if (p == br.end) break;
        // another member follows (anything else fails its header check)
        br.seek(p);
    }
    __syncwarp();
    if (st == STREAM_OK) {
        const uint32_t rest = os.op - os.fp;
        for (uint32_t i = (uint32_t)lane; i < rest; i += 32) os.o[os.fp + i] = w.ring[(os.fp + i) & (IF_RING - 1)];
    }
    if (lane == 0) {
        s.out_len[f] = st == STREAM_OK ? os.op : 0;
        s.status[f] = st;
    }
}

// ------------------------------------------------------------ FASTA records
constexpr int FC_THREADS = 256;
constexpr uint32_t FC_CHUNK = FC_THREADS * 16;  // bytes per round
enum : uint32_t { FS_NONE = 0, FS_SEQ = 1, FS_HDR = 2, FS_FASTQ = 3 };

// Right-most event wins: inclusive scan over the CTA of `v` (FS_NONE = no
// event); returns this thread's exclusive value (`carry` for thread 0) and
// the chunk's last state in *last.
__device__ __forceinline__ uint32_t last_event_scan(uint32_t v, uint32_t carry, uint32_t* sw, uint32_t* last) {
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o && x == FS_NONE) x = y;
    }
    if (lane == 31) sw[wi] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t c = carry;
        for (int i = 0; i < FC_THREADS / 32; ++i) {
            const uint32_t t = sw[i];
            sw[i] = c;  // exclusive state entering warp i
            if (t != FS_NONE) c = t;
        }
        sw[FC_THREADS / 32] = c;
    }
    __syncthreads();
    uint32_t ex = __shfl_up_sync(FULL, x, 1);
    if (lane == 0 || ex == FS_NONE) ex = sw[wi];  // nothing earlier in the warp: the warp's incoming state
    *last = sw[FC_THREADS / 32];
    return ex;
}

__device__ __forceinline__ uint32_t block_sum_excl(uint32_t v, uint32_t* sw, uint32_t* total) {
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sw[wi] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t c = 0;
        for (int i = 0; i < FC_THREADS / 32; ++i) {
            const uint32_t t = sw[i];
            sw[i] = c;
            c += t;
        }
        sw[FC_THREADS / 32] = c;
    }
    __syncthreads();
    const uint32_t r = sw[wi] + x - v;
    *total = sw[FC_THREADS / 32];
    return r;
}

// One CTA per stream, 4 KiB per round.  The record rules (the host reader's
// parse_fasta_fast): the first '>' anywhere starts the first header; a header
// runs to the end of its line; after it, a line starting with '>' starts the
// next record, one starting with '@' or '+' is FASTQ, and every other line is
// sequence (its bytes without the '\n'; empty lines add nothing).  A record's
// '>' is kept as its separator; bytes before the first header are dropped.
__global__ void __launch_bounds__(FC_THREADS) k_fasta_compact(stream_set s, uint64_t* seq_bytes) {
    __shared__ __align__(16) uint8_t chunk[FC_CHUNK];
    __shared__ __align__(16) uint8_t stage[FC_CHUNK + 32];
    __shared__ uint32_t sw[FC_THREADS / 32 + 1], sw2[FC_THREADS / 32 + 1];
    __shared__ uint32_t s_first, s_fastq;
    const uint32_t f = blockIdx.x;
    if (f >= s.n || s.status[f] != STREAM_OK) return;  // whole CTA
    const int t = threadIdx.x;
    uint8_t* base = s.out + s.out_off[f];
    const uint64_t L = s.out_len[f];
    const uint64_t C16 = (s.out_cap[f] + 15) & ~uint64_t(15);
    uint64_t cur = 0, hdrs = 0;
    uint32_t carry_n = 0, state = FS_NONE;
    uint8_t prev = '\n';
    if (t == 0) s_fastq = 0;
    for (uint64_t q = 0; q < L; q += FC_CHUNK) {
        const uint32_t cn = (L - q) < FC_CHUNK ? (uint32_t)(L - q) : FC_CHUNK;
        if (q + 16u * (uint32_t)t < C16)
            reinterpret_cast<uint4*>(chunk)[t] = reinterpret_cast<uint4 const*>(base + q)[t];
        if (t == 0) s_first = FC_CHUNK;
        __syncthreads();
        uint32_t lo = 0;
        if (state == FS_NONE) {
            uint32_t mine = FC_CHUNK;
            for (int j = 0; j < 16; ++j) {
                const uint32_t i = 16u * (uint32_t)t + (uint32_t)j;
                if (i < cn && (chunk[i] == '>' || chunk[i] == '@')) {
                    mine = i;
                    break;
                }
            }
            if (mine < FC_CHUNK) atomicMin(&s_first, mine);
            __syncthreads();
            lo = s_first;
            if (lo == FC_CHUNK) {  // no header yet
                prev = chunk[cn - 1];
                __syncthreads();
                continue;
            }
            if (chunk[lo] == '@') {
                if (t == 0) s_fastq = 1;
                break;
            }
        }
        // events: at lo (the first header) and at line starts after it
        uint32_t ev[16];
        uint32_t tl = FS_NONE;
        for (int j = 0; j < 16; ++j) {
            const uint32_t i = 16u * (uint32_t)t + (uint32_t)j;
            uint32_t e = FS_NONE;
            if (i < cn && i >= lo) {
                const uint8_t b = chunk[i];
                if (state == FS_NONE && i == lo) {
                    e = FS_HDR;
                } else {
                    const uint8_t pb = i ? chunk[i - 1] : prev;
                    if (pb == '\n') e = b == '>' ? FS_HDR : (b == '@' || b == '+') ? FS_FASTQ : FS_SEQ;
                }
            }
            if (e == FS_FASTQ) s_fastq = 1;
            ev[j] = e;
            if (e != FS_NONE) tl = e;
        }
        uint32_t last;
        uint32_t cs = last_event_scan(tl, state, sw, &last);
        uint32_t keep = 0, kc = 0, hc = 0;
        for (int j = 0; j < 16; ++j) {
            const uint32_t i = 16u * (uint32_t)t + (uint32_t)j;
            if (ev[j] != FS_NONE) cs = ev[j];
            const bool k = i < cn && i >= lo &&
                           (ev[j] == FS_HDR || (ev[j] != FS_FASTQ && cs == FS_SEQ && chunk[i] != '\n'));
            keep |= (uint32_t)k << j;
            kc += k;
            hc += ev[j] == FS_HDR;
        }
        uint32_t K;
        const uint32_t at = carry_n + block_sum_excl(kc, sw2, &K);
        uint32_t o = at;
        for (int j = 0; j < 16; ++j)
            if ((keep >> j) & 1u) stage[o++] = chunk[16u * (uint32_t)t + (uint32_t)j];
        // header count of this round (for the sequence-byte total)
        uint32_t H;
        block_sum_excl(hc, sw, &H);
        __syncthreads();
        const uint32_t S = carry_n + K, G = S / 16;
        uint4* dst = reinterpret_cast<uint4*>(base + (cur & ~uint64_t(15)));
        for (uint32_t g = (uint32_t)t; g < G; g += FC_THREADS) dst[g] = reinterpret_cast<uint4 const*>(stage)[g];
        __syncthreads();
        const uint32_t c2 = S - 16 * G;
        uint8_t mv = 0;
        if ((uint32_t)t < c2) mv = stage[16 * G + (uint32_t)t];
        __syncthreads();
        if ((uint32_t)t < c2) stage[t] = mv;
        cur += K;
        hdrs += H;
        carry_n = c2;
        state = last;
        prev = chunk[cn - 1];
        __syncthreads();
        if (s_fastq) break;
    }
    __syncthreads();
    if (s_fastq) {
        if (t == 0) s.status[f] = STREAM_FASTQ;
        return;
    }
    // the partial last group, then '\n' up to the end of the region
    const uint64_t g0 = cur & ~uint64_t(15);
    if (g0 < C16) {
        if ((uint32_t)t < 16 && (uint32_t)t >= carry_n) stage[t] = '\n';
        __syncthreads();
        if (t == 0) *reinterpret_cast<uint4*>(base + g0) = *reinterpret_cast<uint4 const*>(stage);
        const uint4 nl = make_uint4(0x0a0a0a0au, 0x0a0a0a0au, 0x0a0a0a0au, 0x0a0a0a0au);
        for (uint64_t g = g0 + 16 + 16u * (uint64_t)t; g < C16; g += 16u * FC_THREADS)
            *reinterpret_cast<uint4*>(base + g) = nl;
    }
    if (t == 0) {
        s.out_len[f] = cur;
        seq_bytes[f] = cur - hdrs;
    }
}

}  // namespace

void inflate_streams(stream_set const& s, cudaStream_t st) {
    if (!s.n) return;
    k_inflate<<<(s.n + IF_WARPS - 1) / IF_WARPS, IF_WARPS * 32, 0, st>>>(s);
    CDBG_CHECK_LAUNCH();
}

void fasta_compact(stream_set const& s, uint64_t* seq_bytes, cudaStream_t st) {
    if (!s.n) return;
    k_fasta_compact<<<s.n, FC_THREADS, 0, st>>>(s, seq_bytes);
    CDBG_CHECK_LAUNCH();
}

}  // namespace cdbg
