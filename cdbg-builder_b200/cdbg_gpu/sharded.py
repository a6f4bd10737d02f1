"""Builds split across ranks (one GPU per rank).

Phase 2 is bucket-local (the reference's algorithm.md:86-89: a bucket's
graph, walk and color sets need no other bucket), so a build splits into
contiguous bucket ranges: rank r of G builds buckets [B*r/G, B*(r+1)/G) of the
whole collection (cdbg_gpu_build with a bucket range: every rank reads the
input and keeps the super-k-mers of its buckets).  The one exchange step is
the color-set ids: each rank numbers its color sets by first appearance in
its own buckets, the whole build by first appearance over all buckets.  The
shards' fragments and color sets are gathered on one rank in bucket order and
merged there (cdbg_merge_shards): identical sets are recognised by their
encoded bits, new ones appended in order, and the fragments' ids rewritten.
The result is byte for byte the single build's.

The gather goes through torch.distributed (NCCL between GPUs, gloo on CPU).

Phase 1 can also be split, by input file: rank r reads only its consecutive
slice of the files (file_range; colors stay global file indices) and runs
phase 1 on it.  Every rank's bucket records then go to the rank that owns the
bucket (exchange_bucket_records: one all-to-all of the record bytes in bucket
order, whose bucket ranges are contiguous), and the owner merges the records
all ranks made for a bucket into the records one phase 1 over all the files
makes (merge_bucket_records, cdbg_merge_bucket_records) before its phase 2 of
the range.  Nothing is read twice and no minimizer is computed twice."""
import ctypes

import numpy as np

from . import native


def shard_range(num_buckets, rank, world):
    """Buckets [lo, hi) of rank `rank` of `world`."""
    return num_buckets * rank // world, num_buckets * (rank + 1) // world


def merge_shards(shards):
    """shards: [(frag bytes, class words (u64 array), class bits, class offsets
    (u64 array))] in bucket order -> (frag bytes, class words, class offsets)
    of the whole build."""
    L = native.lib()
    n = len(shards)
    frags = [np.frombuffer(s[0], dtype=np.uint8) if len(s[0]) else np.zeros(1, dtype=np.uint8) for s in shards]
    words = [np.ascontiguousarray(s[1], dtype=np.uint64) if len(s[1]) else np.zeros(1, dtype=np.uint64)
             for s in shards]
    offs = [np.ascontiguousarray(s[3], dtype=np.uint64) if len(s[3]) else np.zeros(1, dtype=np.uint64)
            for s in shards]
    vp = ctypes.c_void_p * max(n, 1)
    u64 = ctypes.c_uint64 * max(n, 1)
    fp = vp(*[a.ctypes.data for a in frags])
    fn = u64(*[len(s[0]) for s in shards])
    wp = vp(*[a.ctypes.data for a in words])
    wb = u64(*[int(s[2]) for s in shards])
    op = vp(*[a.ctypes.data for a in offs])
    on = u64(*[len(s[3]) for s in shards])
    m = native.Merged()
    if L.cdbg_merge_shards(n, fp, fn, wp, wb, op, on, ctypes.byref(m)) != 0:
        raise RuntimeError(L.cdbg_merge_last_error().decode(errors="replace"))
    try:
        frag = ctypes.string_at(m.frag_bytes, m.frag_nbytes) if m.frag_nbytes else b""
        nw = (m.class_bits + 63) // 64
        w = (np.ctypeslib.as_array(ctypes.cast(m.class_words, native.c_u64p), shape=(nw,)).copy()
             if nw else np.zeros(0, dtype=np.uint64))
        o = (np.ctypeslib.as_array(ctypes.cast(m.class_offsets, native.c_u64p), shape=(m.n_color_sets,)).copy()
             if m.n_color_sets else np.zeros(0, dtype=np.uint64))
        return frag, w, o, int(m.class_bits)
    finally:
        L.cdbg_merged_free(ctypes.byref(m))


def build_shard(engine, batch, k, num_buckets, num_colors, rank, world, m=0):
    """This rank's share of the build: (frag bytes, class words, class bits,
    class offsets) with its own color-set ids."""
    r = engine.build(batch, k, num_buckets, num_colors, m=m, buckets=shard_range(num_buckets, rank, world))
    return (native.result_frag_bytes(r), native.result_class_words(r), int(r.class_bits),
            native.result_class_offsets(r))


def gather_merge(shard, rank, world, dst=0, group=None):
    """Gather every rank's shard on rank `dst` and merge them there; returns
    the whole build's (frag bytes, class words, class offsets, class bits) on
    `dst` and None elsewhere.  Every rank calls it (a collective)."""
    import torch.distributed as dist
    if world == 1:
        return merge_shards([shard])
    got = [None] * world if rank == dst else None
    dist.gather_object(shard, got, dst=dst, group=group)
    if rank != dst:
        return None
    return merge_shards(got)


def file_range(num_files, rank, world):
    """Input files [lo, hi) that rank `rank` of `world` reads (colors lo..hi-1)."""
    return num_files * rank // world, num_files * (rank + 1) // world


def merge_bucket_records(sources, num_buckets, lo, hi):
    """sources: [(record bytes, offsets of buckets lo..hi (hi - lo + 1))] of
    several ranks' phase 1, in file order -> (bytes, offsets) of the records
    one phase 1 over all their files makes for buckets [lo, hi)."""
    L = native.lib()
    n = len(sources)
    bufs = [np.frombuffer(s[0], dtype=np.uint8) if len(s[0]) else np.zeros(1, dtype=np.uint8) for s in sources]
    offs = [np.ascontiguousarray(s[1], dtype=np.uint64) for s in sources]
    for o in offs:
        if len(o) != hi - lo + 1:
            raise ValueError("each source needs hi - lo + 1 offsets")
    vp = ctypes.c_void_p * max(n, 1)
    m = native.MergedRecords()
    if L.cdbg_merge_bucket_records(n, vp(*[b.ctypes.data for b in bufs]), vp(*[o.ctypes.data for o in offs]),
                                   num_buckets, lo, hi, ctypes.byref(m)) != 0:
        raise RuntimeError(L.cdbg_merge_last_error().decode(errors="replace"))
    try:
        data = ctypes.string_at(m.bytes, m.nbytes) if m.nbytes else b""
        off = np.ctypeslib.as_array(ctypes.cast(m.bucket_off, native.c_u64p), shape=(hi - lo + 1,)).copy()
        return data, off
    finally:
        L.cdbg_merged_records_free(ctypes.byref(m))


def exchange_bucket_records(raw, bucket_off, num_buckets, rank, world, group=None, device="cpu"):
    """raw: this rank's phase-1 records of buckets 0..B-1 back to back,
    bucket_off: their B + 1 offsets.  Sends every rank the records of its
    bucket range (shard_range) and returns, for this rank's range, one
    (bytes, offsets) per source rank, in rank order.  Every rank calls it (two
    all-to-alls: the offsets, then the bytes; NCCL needs device="cuda")."""
    import torch
    import torch.distributed as dist
    bucket_off = np.asarray(bucket_off, dtype=np.int64)
    rng = [shard_range(num_buckets, q, world) for q in range(world)]
    lo, hi = rng[rank]
    if world == 1:
        return [(bytes(raw), (bucket_off[lo:hi + 1] - bucket_off[lo]).astype(np.uint64))]
    # per destination: its buckets' offsets, relative to the start of its bytes
    off_send = np.concatenate([bucket_off[a:b + 1] - bucket_off[a] for a, b in rng])
    off_in = [b - a + 1 for a, b in rng]
    off_out = [hi - lo + 1] * world
    t_off = torch.empty(sum(off_out), dtype=torch.int64, device=device)
    dist.all_to_all_single(t_off, torch.from_numpy(off_send).to(device), off_out, off_in, group=group)
    offs = t_off.cpu().numpy().reshape(world, hi - lo + 1)
    byte_in = [int(bucket_off[b] - bucket_off[a]) for a, b in rng]
    byte_out = [int(offs[s][-1]) for s in range(world)]
    send = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy() if len(raw) else np.zeros(0, np.uint8))
    t_bytes = torch.empty(sum(byte_out), dtype=torch.uint8, device=device)
    dist.all_to_all_single(t_bytes, send.to(device), byte_out, byte_in, group=group)
    got = t_bytes.cpu().numpy().tobytes()
    out, p = [], 0
    for s in range(world):
        out.append((got[p:p + byte_out[s]], offs[s].astype(np.uint64)))
        p += byte_out[s]
    return out


def read_bucket_dir(d, num_buckets):
    """This rank's phase-1 bucket files (bucket_<b>.bin in d, a missing file an
    empty bucket), decompressed: (record bytes of buckets 0..B-1, B + 1 offsets)."""
    import os
    from . import formats
    parts, off = [], np.zeros(num_buckets + 1, dtype=np.uint64)
    for b in range(num_buckets):
        p = os.path.join(d, "bucket_%d.bin" % b)
        raw = formats.read_bucket_raw(p) if os.path.exists(p) else b""
        parts.append(raw)
        off[b + 1] = off[b] + len(raw)
    return b"".join(parts), off


def write_bucket_dir(d, lo, data, off):
    """Bucket files lo.. of merged records (one LZ4 frame each) in d."""
    import os
    from . import formats
    os.makedirs(d, exist_ok=True)
    for i in range(len(off) - 1):
        formats.write_bucket_raw(os.path.join(d, "bucket_%d.bin" % (lo + i)), data[int(off[i]):int(off[i + 1])])


def shard_from_phase2(frag_path, color_sets_path):
    """(frag bytes, class words, class bits, class offsets) of a drop-in
    phase 2's two files."""
    from . import formats
    frag = open(frag_path, "rb").read()
    _, words, offs, _ = formats.read_color_sets(color_sets_path, decode=False)
    bits = int(np.fromfile(color_sets_path, dtype=np.uint64, count=1, offset=12)[0])
    return frag, np.asarray(words, dtype=np.uint64), bits, np.asarray(offs, dtype=np.uint64)


def build_rank_by_files(engine, files, k, num_buckets, rank, world, work_dir, group=None, device="cuda", m=0):
    """This rank's part of a build split by input file: the drop-in phase 1
    of its slice of the files, the record exchange and merge, the drop-in
    phase 2 of its bucket range.  Returns its shard for gather_merge.  Every
    rank calls it (the exchange is a collective)."""
    import os
    f0, f1 = file_range(len(files), rank, world)
    p1 = os.path.join(work_dir, "p1")
    engine.phase1(files[f0:f1], k, num_buckets, p1, m=m, first_color=f0)
    raw, off = read_bucket_dir(p1, num_buckets)
    got = exchange_bucket_records(raw, off, num_buckets, rank, world, group=group, device=device)
    lo, hi = shard_range(num_buckets, rank, world)
    data, moff = merge_bucket_records(got, num_buckets, lo, hi)
    md = os.path.join(work_dir, "merged")
    write_bucket_dir(md, lo, data, moff)
    frag, cs = os.path.join(work_dir, "frag_unitigs.bin"), os.path.join(work_dir, "out.color_sets")
    engine.phase2(md, num_buckets, k, len(files), frag, cs)
    return shard_from_phase2(frag, cs)


# ---- color-set interning across ranks -----------------------------------------
# gather_merge interns every shard's classes on one rank.  intern_classes does
# it hash-partitioned instead: the owner of a class (its hash mod the ranks)
# learns every (rank, local id) that has it and which rank saw it first (the
# lowest rank: buckets are split in rank order); each rank numbers the classes
# it saw first in its own order, after the ranks before it (a prefix sum of
# their counts), which is the single build's first-appearance order over
# buckets 0..B-1; the owners pass those ids to the other holders, and every
# rank rewrites its own fragments.  No rank holds more than its share of the
# classes, and only the classes each rank saw first make up the .color_sets
# bit vector.

def _all_to_all_bytes(blobs, world, group=None, device="cpu"):
    """blobs[q] goes to rank q; returns what every rank sent here, in rank order."""
    import torch
    import torch.distributed as dist
    sizes = torch.tensor([len(b) for b in blobs], dtype=torch.int64, device=device)
    got_sizes = torch.empty(world, dtype=torch.int64, device=device)
    dist.all_to_all_single(got_sizes, sizes, group=group)
    got_sizes = [int(x) for x in got_sizes.cpu().tolist()]
    cat = b"".join(blobs)
    send = torch.from_numpy(np.frombuffer(cat, dtype=np.uint8).copy() if cat else np.zeros(0, np.uint8))
    recv = torch.empty(sum(got_sizes), dtype=torch.uint8, device=device)
    dist.all_to_all_single(recv, send.to(device), got_sizes, [len(b) for b in blobs], group=group)
    data = recv.cpu().numpy().tobytes()
    out, p = [], 0
    for n in got_sizes:
        out.append(data[p:p + n])
        p += n
    return out


def class_strings(words, class_bits, offsets):
    """(hashes, strings, string offsets): each class's bits from bit 0 in whole
    words and its 64-bit hash (cdbg_class_strings)."""
    L = native.lib()
    n = len(offsets)
    w = np.ascontiguousarray(words, dtype=np.uint64) if len(words) else np.zeros(1, dtype=np.uint64)
    o = np.ascontiguousarray(offsets, dtype=np.uint64) if n else np.zeros(1, dtype=np.uint64)
    hashes = np.zeros(max(n, 1), dtype=np.uint64)
    cap = int(class_bits) // 64 + n + 1
    strings = np.zeros(cap, dtype=np.uint64)
    soff = np.zeros(n + 1, dtype=np.uint64)
    if L.cdbg_class_strings(w.ctypes.data, int(class_bits), o.ctypes.data, n, hashes.ctypes.data,
                            strings.ctypes.data, cap, soff.ctypes.data) != 0:
        raise RuntimeError(L.cdbg_merge_last_error().decode(errors="replace"))
    return hashes[:n], strings, soff


def remap_frag(frag, mapping):
    """frag bytes with their color-set ids rewritten through `mapping`."""
    L = native.lib()
    buf = bytearray(frag)
    m = np.ascontiguousarray(mapping, dtype=np.uint64) if len(mapping) else np.zeros(1, dtype=np.uint64)
    cb = (ctypes.c_char * len(buf)).from_buffer(buf) if buf else None
    if L.cdbg_frag_remap_classes(ctypes.addressof(cb) if cb is not None else None, len(buf), m.ctypes.data,
                                 len(mapping)) != 0:
        raise RuntimeError(L.cdbg_merge_last_error().decode(errors="replace"))
    return bytes(buf)


def intern_classes(shard, rank, world, group=None, device="cpu"):
    """shard: (frag bytes, class words, class bits, class offsets) of this
    rank's bucket range, ranks in bucket order.  Returns (frag bytes with the
    whole build's color-set ids, the bit strings of the classes this rank saw
    first as (words, bits), their lengths in bits, the whole-build id of the
    first of them).  Every rank calls it (a collective)."""
    import pickle
    import torch
    import torch.distributed as dist
    frag, words, bits, offs = shard
    n = len(offs)
    hashes, strings, soff = class_strings(words, bits, offs)
    lens = [int(offs[c + 1] if c + 1 < n else bits) - int(offs[c]) for c in range(n)]

    def key(c):
        return lens[c], strings[int(soff[c]):int(soff[c + 1])].tobytes()

    # 1. every class to its owner
    out = [[] for _ in range(world)]
    for c in range(n):
        ln, s = key(c)
        out[int(hashes[c]) % world].append((c, ln, s))
    got = [pickle.loads(b) for b in _all_to_all_bytes([pickle.dumps(x) for x in out], world, group, device)]
    # 2. the owner finds each class's first holder and tells every holder
    first = {}
    for src in range(world):  # rank order: the first holder is the lowest rank
        for c, ln, s in got[src]:
            first.setdefault((ln, s), (src, c))
    reply = [[(c, first[(ln, s)]) for c, ln, s in got[src]] for src in range(world)]
    back = [pickle.loads(b) for b in _all_to_all_bytes([pickle.dumps(x) for x in reply], world, group, device)]
    firsts = [None] * n
    for part in back:
        for c, f in part:
            firsts[c] = f
    new = [c for c in range(n) if firsts[c] == (rank, c)]
    # 3. ids: the classes this rank saw first, after those of the ranks before it
    counts = [0] * world
    dist.all_gather_object(counts, len(new), group=group)
    base = sum(counts[:rank])
    gid = np.full(n, np.iinfo(np.uint64).max, dtype=np.uint64)
    for i, c in enumerate(new):
        gid[c] = base + i
    # 4. the owners pass the new ids to every holder
    tell = [[] for _ in range(world)]
    for c in new:
        tell[int(hashes[c]) % world].append((c, int(gid[c])))
    learned = [pickle.loads(b) for b in _all_to_all_bytes([pickle.dumps(x) for x in tell], world, group, device)]
    first_gid = {}
    for src in range(world):
        for c, g in learned[src]:
            first_gid[(src, c)] = g
    answer = [[(c, first_gid[first[(ln, s)]]) for c, ln, s in got[src]] for src in range(world)]
    final = [pickle.loads(b) for b in _all_to_all_bytes([pickle.dumps(x) for x in answer], world, group, device)]
    for part in final:
        for c, g in part:
            gid[c] = g
    # 5. this rank's fragments and its classes' bits
    seg = _concat_bits([(strings[int(soff[c]):int(soff[c + 1])], lens[c]) for c in new])
    return remap_frag(frag, gid), seg, [lens[c] for c in new], base


def _concat_bits(parts):
    """[(words from bit 0, nbits)] -> (words, nbits) of the bit strings back to back."""
    total = sum(int(nb) for _, nb in parts)
    out = np.zeros((total + 63) // 64 + 1, dtype=np.uint64)
    pos = 0
    for w, nb in parts:
        nb = int(nb)
        if nb == 0:
            continue
        nw = (nb + 63) // 64
        w = np.array(w[:nw], dtype=np.uint64)
        if nb % 64:
            w[-1] &= np.uint64((1 << (nb % 64)) - 1)
        i, s = pos // 64, pos % 64
        if s == 0:
            out[i:i + nw] |= w
        else:
            out[i:i + nw] |= w << np.uint64(s)
            out[i + 1:i + nw + 1] |= w >> np.uint64(64 - s)
        pos += nb
    return out[:(total + 63) // 64], total


def assemble(interned, rank, world, dst=0, group=None):
    """The whole build's (frag bytes, class words, class offsets, class bits)
    on rank `dst` (None elsewhere) from every rank's intern_classes result:
    the fragments and the class bit strings back to back in rank order, the
    class offsets from the strings' lengths."""
    import torch.distributed as dist
    got = [None] * world if rank == dst else None
    dist.gather_object(interned, got, dst=dst, group=group)
    if rank != dst:
        return None
    frag = b"".join(g[0] for g in got)
    words, bits = _concat_bits([g[1] for g in got])
    lens = [ln for g in got for ln in g[2]]
    offsets = np.zeros(len(lens), dtype=np.uint64)
    if lens:
        offsets[1:] = np.cumsum(np.asarray(lens[:-1], dtype=np.uint64))
    return frag, words, offsets, bits
