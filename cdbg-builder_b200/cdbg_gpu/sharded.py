"""Builds split by bucket range across ranks (one GPU per rank).

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

The gather goes through torch.distributed (NCCL between GPUs, gloo on CPU)."""
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
