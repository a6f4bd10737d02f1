"""Readers for the on-disk artifacts of phases 1 and 2 (inspection and parity).

* bucket files   ``bucket_<b>.bin``: LZ4 frames ``[u32 unc][u32 comp][bytes]``,
                 ``[u32 0]`` end marker (bucket_io.hpp:19-40); records
                 ``varint ncolors, varint color deltas, varint (len<<4|flags),
                 packed bases`` (super_kmer.hpp:1-29, 105-143).
* frag spill     ``frag_unitigs.bin``: ``[u8 open][u32 nruns][nruns x (u64 cid,
                 u32 num_kmers)][u32 seq_len][seq]`` (unitig_spill.hpp:642-665).
* .color_sets    ``[u32 C][u32 sparse][u32 dense][u64 bits][u64 words][words]``
                 then Elias-Fano of the class offsets
                 (streaming_color_set_dict.hpp:29-37, 221-294); classes are
                 hybrid-encoded (hybrid_color_sets.hpp:48-95) with
                 delta(x) = Elias delta of x + 1, LSB-first.
"""
import ctypes
import struct

import numpy as np

FOREIGN = (1 << 64) - 1

_lz4 = None


def _lz4lib():
    global _lz4
    if _lz4 is None:
        _lz4 = ctypes.CDLL("liblz4.so.1")
        _lz4.LZ4_decompress_safe.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        _lz4.LZ4_decompress_safe.restype = ctypes.c_int
        _lz4.LZ4_compressBound.argtypes = [ctypes.c_int]
        _lz4.LZ4_compressBound.restype = ctypes.c_int
        _lz4.LZ4_compress_default.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        _lz4.LZ4_compress_default.restype = ctypes.c_int
    return _lz4


def write_bucket_raw(path, raw):
    """A bucket file (bucket_io.hpp:19-40 frames) holding `raw` record bytes
    in one LZ4 frame, then the end mark."""
    L = _lz4lib()
    with open(path, "wb") as f:
        if raw:
            cap = L.LZ4_compressBound(len(raw))
            dst = ctypes.create_string_buffer(cap)
            c = L.LZ4_compress_default(bytes(raw), dst, len(raw), cap)
            if c <= 0:
                raise RuntimeError("LZ4_compress_default failed on " + path)
            f.write(struct.pack("<II", len(raw), c) + dst.raw[:c])
        f.write(struct.pack("<I", 0))


def read_bucket_raw(path):
    """Decompressed record bytes of one bucket file."""
    out = bytearray()
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p + 4 <= len(data):
        (u,) = struct.unpack_from("<I", data, p)
        p += 4
        if u == 0:
            break
        (c,) = struct.unpack_from("<I", data, p)
        p += 4
        dst = ctypes.create_string_buffer(u)
        d = _lz4lib().LZ4_decompress_safe(bytes(data[p:p + c]), dst, c, u)
        if d != u:
            raise RuntimeError("LZ4_decompress_safe failed on " + path)
        out += dst.raw
        p += c
    return bytes(out)


def _varint(b, p):
    v = 0
    s = 0
    while True:
        c = b[p]
        p += 1
        v |= (c & 0x7F) << s
        if not c & 0x80:
            return v, p
        s += 7


def parse_records(raw):
    """[(flags, colors tuple, bases 'ACGT' string)] of a decompressed bucket."""
    out = []
    p = 0
    while p < len(raw):
        n, p = _varint(raw, p)
        cols = []
        prev = 0
        for _ in range(n):
            d, p = _varint(raw, p)
            prev += d
            cols.append(prev)
        lf, p = _varint(raw, p)
        ln, fl = lf >> 4, lf & 15
        nb = (ln + 3) // 4
        chunk = raw[p:p + nb]
        p += nb
        bases = "".join("ACGT"[(chunk[i >> 2] >> (2 * (i & 3))) & 3] for i in range(ln))
        out.append((fl, tuple(cols), bases))
    return out


def read_frags(data):
    """[(open_flags, [(cid, num_kmers)], seq)] from frag spill bytes or a path."""
    if isinstance(data, str):
        with open(data, "rb") as f:
            data = f.read()
    out = []
    p = 0
    n = len(data)
    while p < n:
        fl = data[p]
        (nr,) = struct.unpack_from("<I", data, p + 1)
        p += 5
        runs = []
        for _ in range(nr):
            cid, nk = struct.unpack_from("<QI", data, p)
            runs.append((cid, nk))
            p += 12
        (sl,) = struct.unpack_from("<I", data, p)
        p += 4
        out.append((fl, runs, data[p:p + sl].decode()))
        p += sl
    return out


class _Bits:
    def __init__(self, words, pos):
        self.w = words
        self.p = pos

    def take(self, n):
        v = 0
        for i in range(n):
            q = self.p + i
            v |= ((int(self.w[q >> 6]) >> (q & 63)) & 1) << i
        self.p += n
        return v

    def zeros(self):
        z = 0
        while not (int(self.w[self.p >> 6]) >> (self.p & 63)) & 1:
            z += 1
            self.p += 1
        return z


def read_gamma(b):
    l = b.zeros()
    b.take(1)
    return (1 << l) | b.take(l)


def read_delta(b):
    l = read_gamma(b) - 1
    return ((1 << l) | b.take(l)) - 1


def decode_class(words, pos, C):
    """Inverse of the hybrid encoder at bit `pos` (compact_color_set_dict.hpp:176-222)."""
    sparse_t, dense_t = int(0.25 * C), int(0.75 * C)
    b = _Bits(words, pos)
    N = read_delta(b)
    if N == 0:
        return []
    if N < sparse_t:
        prev = read_delta(b)
        out = [prev]
        for _ in range(1, N):
            prev = prev + read_delta(b) + 1
            out.append(prev)
        return out
    if N < dense_t:
        return [i for i in range(C) if b.take(1)]
    comp = C - N
    absent = set()
    if comp:
        prev = read_delta(b)
        absent.add(prev)
        for _ in range(1, comp):
            prev = prev + read_delta(b) + 1
            absent.add(prev)
    return [v for v in range(C) if v not in absent]


def ef_values(low, high, n, l):
    """The n values of an Elias-Fano sequence (l low bits each), vectorized."""
    bits = np.unpackbits(np.asarray(high, dtype=np.uint64).view(np.uint8), bitorder="little")
    pos = np.flatnonzero(bits)[:n].astype(np.uint64)
    hi = pos - np.arange(len(pos), dtype=np.uint64)
    if l == 0:
        return hi
    q = np.arange(len(pos), dtype=np.uint64) * np.uint64(l)
    w = (q >> np.uint64(6)).astype(np.int64)
    sh = q & np.uint64(63)
    lw = np.append(np.asarray(low, dtype=np.uint64), np.uint64(0))
    v = lw[w] >> sh
    spill = sh + np.uint64(l) > np.uint64(64)
    nxt = np.where(spill, lw[np.minimum(w + 1, len(lw) - 1)] << ((np.uint64(64) - sh) & np.uint64(63)),
                   np.uint64(0))
    lo = (v | nxt) & np.uint64((1 << l) - 1)
    return (hi << np.uint64(l)) | lo


def read_color_sets(path, decode=True):
    """(C, words ndarray, class offsets list, decoded classes list, or None
    without decode)."""
    with open(path, "rb") as f:
        data = f.read()
    C, st, dt, nbits, nwords = struct.unpack_from("<IIIQQ", data, 0)
    p = 28
    words = np.frombuffer(data, dtype=np.uint64, count=nwords, offset=p).copy() if nwords else \
        np.zeros(1, dtype=np.uint64)
    p += 8 * nwords
    U, n, l = struct.unpack_from("<QQQ", data, p)
    p += 24
    lb, lw = struct.unpack_from("<QQ", data, p)
    p += 16
    low = np.frombuffer(data, dtype=np.uint64, count=lw, offset=p) if lw else np.zeros(0, np.uint64)
    p += 8 * lw
    hb, hw = struct.unpack_from("<QQ", data, p)
    p += 16
    high = np.frombuffer(data, dtype=np.uint64, count=hw, offset=p) if hw else np.zeros(0, np.uint64)
    offs = [int(x) for x in ef_values(low, high, n, l)]
    offsets = offs[:-1]
    if nwords == 0:
        words = np.zeros(1, dtype=np.uint64)
    classes = [decode_class(np.append(words, np.uint64(0)), o, C) for o in offsets] if decode else None
    return C, words[:nwords], offsets, classes


def decode_classes(words, offsets, C):
    w = np.append(np.asarray(words, dtype=np.uint64), np.uint64(0))
    return [decode_class(w, int(o), C) for o in offsets]


_RC = str.maketrans("ACGT", "TGCA")


def revcomp(s):
    return s.translate(_RC)[::-1]


def canonical_frag(fl, runs, seq, classes):
    """Orientation-free form of a fragment: (seq, per-k-mer color sets, open bits)
    taken in whichever orientation has the smaller sequence; cids are replaced
    by their decoded color sets so different id orders compare equal."""
    per = []
    for cid, nk in runs:
        cs = None if cid == FOREIGN else tuple(classes[cid])
        per.extend([cs] * nk)
    rs = revcomp(seq)
    if rs < seq:
        return (rs, tuple(reversed(per)), ((fl & 1) << 1) | ((fl >> 1) & 1))
    return (seq, tuple(per), fl)


# ---- final outputs (.fa, .metadata.txt) written by phases 3 and 4 ----------

def write_classes(path, classes):
    """Class list file read by the phase-3/4 runner: u64 count, then per class
    u32 n and n ascending u32 colors."""
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(classes)))
        for c in classes:
            f.write(struct.pack("<I", len(c)))
            if len(c):
                f.write(np.asarray(c, dtype=np.uint32).tobytes())


def read_fasta_unitigs(path):
    """[(cid, seq)] of a phase-4 .fa (`>cid` headers, emit.hpp:93-175)."""
    out = []
    cid = None
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if line.startswith(">"):
                cid = int(line[1:].split()[0])
            elif line:
                out.append((cid, line))
    return out


def read_metadata(path):
    """key -> int of a .metadata.txt (builder.hpp:754-764)."""
    d = {}
    with open(path) as f:
        for line in f:
            if "=" in line:
                key, v = line.strip().split("=", 1)
                d[key] = int(v)
    return d


def canonical_unitig(seq, k):
    """Orientation- and rotation-free form of a unitig.  A unitig whose last
    k-1 bases repeat its first k-1 may be a cycle, whose starting k-mer is
    arbitrary: it is replaced by the smallest rotation of its k-mer cycle over
    both strands (rotations of one k-mer cycle never belong to two different
    unitigs of one build, so this cannot merge distinct unitigs)."""
    rs = revcomp(seq)
    if len(seq) > k - 1 and k > 1 and seq[-(k - 1):] == seq[:k - 1]:
        best = None
        for s in (seq, rs):
            core = s[:len(s) - (k - 1)]
            n = len(core)
            for r in range(n):
                rot = core[r:] + core[:r]
                cand = rot + rot[:k - 1]
                if best is None or cand < best:
                    best = cand
        return best
    return min(seq, rs)


def final_pairs(basename, k):
    """Multiset of (canonical unitig, decoded color set) of a finished build,
    its metadata and its color-set family."""
    from collections import Counter
    _, _, _, classes = read_color_sets(basename + ".color_sets")
    pairs = Counter((canonical_unitig(s, k), tuple(classes[c])) for c, s in read_fasta_unitigs(basename + ".fa"))
    return pairs, read_metadata(basename + ".metadata.txt"), Counter(tuple(c) for c in classes)
