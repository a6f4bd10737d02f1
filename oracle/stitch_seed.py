"""CPU restatement of the stitch's round-0 seed -- test infrastructure only.

The checker for cdbg_gpu_stitch_seed: pure Python, for inputs of a few MB.
It restates, from the reference (paths relative to its repository):

  ext_seed_one                  phase3_stitch/stitch_extmem.hpp:930-944
  ext_seed_from_seq (FNV-1a)    :244-251
  ext_mix_bit (splitmix64 top)  :233-240
  ext_choose_side               :287-304
  side_kmer_canonical           :261-274
  ext_route                     :609-620 with kmer_hasher (kmer.hpp:127-149)
  ext_tig_serialize             :407-428
  ext_split_monochromatic       :113-150
  round_store_file emit/flush   :497-501, :572-597 (4 MiB frames)

and the frag record layout of frag_unitig_writer (phase2_bucket_process/
unitig_spill.hpp:491-522).  It is pinned against the reference's own seed
(oracle/_ref/ref_seed, built from the reference's sources) by
tests/test_seed_oracle.py.
"""
import struct

M64 = (1 << 64) - 1
FOREIGN = M64                 # COLOR_RUN_FOREIGN (bucket_walker.hpp:96)
OPEN_LEFT, OPEN_RIGHT = 1, 2  # UNITIG_OPEN_* (bucket_walker.hpp:80-81)
FRAME = 4 << 20               # round_store_file::FRAME_BUDGET (stitch_extmem.hpp:556)
CODE = {ord("A"): 0, ord("a"): 0, ord("C"): 1, ord("c"): 1, ord("G"): 2, ord("g"): 2, ord("T"): 3, ord("t"): 3}


def parse_frags(buf):
    """frag_unitigs.bin -> [(open_flags, [(cid, num_kmers)], seq bytes)]."""
    out, p, n = [], 0, len(buf)
    while p < n:
        of = buf[p]
        (nr,) = struct.unpack_from("<I", buf, p + 1)
        runs = [struct.unpack_from("<QI", buf, p + 5 + 12 * i) for i in range(nr)]
        lp = p + 5 + 12 * nr
        (ln,) = struct.unpack_from("<I", buf, lp)
        out.append((of, runs, bytes(buf[lp + 4:lp + 4 + ln])))
        p = lp + 4 + ln
    return out


def frag_record(of, runs, seq):
    b = bytearray(struct.pack("<BI", of, len(runs)))
    for cid, m in runs:
        b += struct.pack("<QI", cid, m)
    b += struct.pack("<I", len(seq)) + seq
    return bytes(b)


def seed_from_seq(seq):
    h = 1469598103934665603
    for c in seq:
        h = ((h ^ c) * 1099511628211) & M64
    return h if h else 0x9E3779B97F4A7C15


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def kmer_hash(x, wide):
    if not wide:
        return mix64(x & M64)
    lo, hi = x & M64, x >> 64
    return (mix64(lo) ^ ((mix64((hi + 0x9E3779B97F4A7C15) & M64) << 1) & M64)) & M64


def side_kmer_canonical(seq, k, right):
    p = seq[len(seq) - k:] if right else seq[:k]
    fwd = 0
    for c in p:
        fwd = (fwd << 2) | CODE[c]
    rc = 0
    x = fwd
    for _ in range(k):
        rc = (rc << 2) | (3 - (x & 3))
        x >>= 2
    return fwd if fwd <= rc else rc


def tig_bytes(of, rng, runs, seq):
    b = bytearray(struct.pack("<BQI", of, rng, len(runs)))
    for cid, m in runs:
        b += struct.pack("<QI", cid, m)
    b += struct.pack("<I", len(seq))
    packed = bytearray((len(seq) + 3) // 4)
    for i, c in enumerate(seq):
        packed[i >> 2] |= (CODE.get(c, 0xFF) << (2 * (i & 3))) & 0xFF
    return bytes(b + packed)


def split_monochromatic(runs, seq, k, of):
    lo, hi = 0, len(runs)
    if lo < hi and runs[lo][0] == FOREIGN:
        lo += 1
    if lo < hi and runs[hi - 1][0] == FOREIGN:
        hi -= 1
    base = sum(m for _, m in runs[:lo])
    out = []
    for i in range(lo, hi):
        cid, m = runs[i]
        if cid == FOREIGN:
            base += m
            continue
        if base > len(seq):
            raise ValueError("substr past the end")
        piece = seq[base:base + m + k - 1]
        f = (of & OPEN_LEFT if i == lo else 0) | (of & OPEN_RIGHT if i + 1 == hi else 0)
        out.append(frag_record(f, [(cid, m)], piece))
        base += m
    return out


def seed(frag_buf, k, num_buckets, wide=None):
    """Round 0 of a one-thread seed: per bucket, the list of frames (raw,
    uncompressed bytes) its round-0 file holds, and the closed unitigs' frag
    records back to back."""
    if wide is None:
        wide = k > 31
    batch = [bytearray() for _ in range(num_buckets)]
    frames = [[] for _ in range(num_buckets)]
    closed = bytearray()
    for of, runs, seq in parse_frags(frag_buf):
        rng = seed_from_seq(seq)
        if k < 2 or of == 0:
            for r in split_monochromatic(runs, seq, k, of):
                closed += r
            continue
        both = (of & OPEN_LEFT) and (of & OPEN_RIGHT)
        right = bool(mix64(rng) >> 63) if both else not (of & OPEN_LEFT)
        j = side_kmer_canonical(seq, k, right)
        b = (kmer_hash(j, wide) >> 1) % num_buckets
        batch[b] += tig_bytes(of, rng, runs, seq)
        if len(batch[b]) >= FRAME:
            frames[b].append(bytes(batch[b]))
            batch[b] = bytearray()
    for b in range(num_buckets):
        if batch[b]:
            frames[b].append(bytes(batch[b]))
    return frames, bytes(closed)
