"""CPU: phase 1 split by input file.  Each rank runs phase 1 on its own slice
of the files only (colors stay global file indices); the bucket records go to
the rank that owns the bucket (one all-to-all over torch.distributed, gloo,
world size 2, two processes), which merges them into the records one phase 1
over all the files makes, then runs phase 2 of its bucket range; the shards
are gathered and merged on one rank.  The records and the final outputs equal
the single build's byte for byte, merged on one rank or with the color sets
interned across the ranks.

Phase 1 and phase 2 of each rank are made here by the CPU oracle, in the
places the GPU drop-in phases run on a rank's GPU; what is under test is the
product's exchange and merges (cdbg_gpu/sharded.py, cdbg_merge_bucket_records,
cdbg_merge_shards)."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, ORACLE_LIB

K, B, N = 31, 64, 6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _collection(d, seed=31):
    from cdbg_gpu import synth
    p = synth.make_params(seed=seed, len_min=20000, len_max=60000, div_min=0.002, div_max=0.02, indels=5,
                          mobile_pool=2, mobile_min=500, mobile_max=1500, contigs_min=1, contigs_max=8,
                          contigs_log=1, lowercase_runs=1, n_runs=1)
    lst = synth.write_fasta(p, N, os.path.join(d, "in"))
    return [l.strip() for l in open(lst) if l.strip()]


def _phase1(files, first_color, out_dir):
    """The oracle's phase 1 of `files` read as colors first_color.. into bucket files."""
    L = ctypes.CDLL(ORACLE_LIB)
    L.oracle_phase1_from.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
    L.oracle_last_error.restype = ctypes.c_char_p
    os.makedirs(out_dir, exist_ok=True)
    lst = os.path.join(out_dir, "files.txt")
    with open(lst, "w") as f:
        f.write("".join(x + "\n" for x in files))
    if L.oracle_phase1_from(lst.encode(), first_color, K, 0, B, None, out_dir.encode(), None, None) != 0:
        raise RuntimeError(L.oracle_last_error().decode())


def _phase2_shard(orc, bucket_dir, out):
    """(frag bytes, class words, class bits, class offsets) of the oracle's phase 2."""
    from cdbg_gpu import formats
    orc.phase2(bucket_dir, B, K, N, out)
    frag = open(os.path.join(out, "frag_unitigs.bin"), "rb").read()
    _, words, offs, _ = formats.read_color_sets(os.path.join(out, "out.color_sets"))
    bits = int(np.fromfile(os.path.join(out, "out.color_sets"), dtype=np.uint64, count=1, offset=12)[0])
    return frag, np.asarray(words, dtype=np.uint64), bits, np.asarray(offs, dtype=np.uint64)


def _worker(rank, world, port, d, out):
    import sys
    for p in (ROOT, os.path.join(ROOT, "cdbg-builder_b200"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    from conftest import Oracle
    from cdbg_gpu import sharded
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                           timeout=datetime.timedelta(seconds=60))
    try:
        files = [l.strip() for l in open(os.path.join(d, "in", "filenames.txt")) if l.strip()]
        rd = os.path.join(d, "rank%d" % rank)
        f0, f1 = sharded.file_range(len(files), rank, world)
        _phase1(files[f0:f1], f0, os.path.join(rd, "p1"))
        raw, off = sharded.read_bucket_dir(os.path.join(rd, "p1"), B)
        got = sharded.exchange_bucket_records(raw, off, B, rank, world)
        lo, hi = sharded.shard_range(B, rank, world)
        data, moff = sharded.merge_bucket_records(got, B, lo, hi)
        sharded.write_bucket_dir(os.path.join(rd, "merged"), lo, data, moff)
        shard = _phase2_shard(Oracle(), os.path.join(rd, "merged"), os.path.join(rd, "out"))
        whole = sharded.gather_merge(shard, rank, world)
        # the same shards interned across the ranks instead of on one
        spread = sharded.assemble(sharded.intern_classes(shard, rank, world), rank, world)
        recs = (lo, data, moff.tobytes())
        allrecs = [None] * world if rank == 0 else None
        dist.gather_object(recs, allrecs, dst=0)
        if rank == 0:
            frag, w, o, bits = whole
            assert spread[0] == frag and spread[1].tobytes() == w.tobytes()
            assert spread[2].tobytes() == o.tobytes() and spread[3] == bits
            out.put((frag, w.tobytes(), o.tobytes(), bits, allrecs))
    finally:
        dist.destroy_process_group()


def _single(d, files):
    from conftest import Oracle
    from cdbg_gpu import sharded
    sd = os.path.join(d, "single")
    _phase1(files, 0, os.path.join(sd, "p1"))
    raw, off = sharded.read_bucket_dir(os.path.join(sd, "p1"), B)
    return raw, off, _phase2_shard(Oracle(), os.path.join(sd, "p1"), os.path.join(sd, "out"))


def test_two_ranks_split_by_file_equal_the_single_build(tmp_path):
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built")
    d = str(tmp_path)
    files = _collection(d)
    raw, off, want = _single(d, files)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, d, q)) for r in range(2)]
    for p in procs:
        p.start()
    frag, w, o, bits, allrecs = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every bucket's merged records are the single phase 1's
    for lo, data, moff in allrecs:
        moff = np.frombuffer(moff, dtype=np.uint64)
        for i in range(len(moff) - 1):
            b = lo + i
            assert data[int(moff[i]):int(moff[i + 1])] == raw[int(off[b]):int(off[b + 1])], b
    assert frag == want[0]
    assert w == want[1].tobytes() and bits == want[2]
    assert o == want[3].tobytes()


@pytest.mark.parametrize("slices", [[0, 6], [0, 1, 6], [0, 2, 3, 6], [0, 1, 2, 3, 4, 5, 6]])
def test_merge_of_file_slices_is_the_single_phase1(tmp_path, slices):
    """Any split of the files into consecutive slices (several per source too:
    a rank whose phase 1 ran in chunks holds one sorted run per chunk) merges
    to the single phase 1's records."""
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built")
    from cdbg_gpu import sharded
    d = str(tmp_path)
    files = _collection(d, seed=37)
    raw, off, _ = _single(d, files)
    runs = []
    for i in range(len(slices) - 1):
        sd = os.path.join(d, "s%d" % i)
        _phase1(files[slices[i]:slices[i + 1]], slices[i], sd)
        runs.append(sharded.read_bucket_dir(sd, B))
    # sources: the slices one by one, and the slices paired into "chunked" sources
    one = [(r, o) for r, o in runs]
    paired = []
    for i in range(0, len(runs), 2):
        grp = runs[i:i + 2]
        parts, po = [], np.zeros(B + 1, dtype=np.uint64)
        for b in range(B):
            chunk = b"".join(r[int(o[b]):int(o[b + 1])] for r, o in grp)
            parts.append(chunk)
            po[b + 1] = po[b] + len(chunk)
        paired.append((b"".join(parts), po))
    for srcs in (one, paired):
        for lo, hi in ((0, B), (5, 40)):
            sources = [(r, (o[lo:hi + 1] - o[lo]).astype(np.uint64)) for r, o in srcs]
            sources = [(r[int(o0[lo]):int(o0[hi])], so) for (r, so), (_, o0) in zip(sources, srcs)]
            data, moff = sharded.merge_bucket_records(sources, B, lo, hi)
            assert data == raw[int(off[lo]):int(off[hi])]
            assert np.array_equal(moff, (off[lo:hi + 1] - off[lo]).astype(np.uint64))


def test_merge_and_remap_reject_malformed_input():
    """Truncated records, bad ranges and ids past the map are errors, not
    wrong output."""
    from cdbg_gpu import native, sharded
    # one record: 1 color (7), len 5 flags 3, 2 bytes of bases
    rec = bytes([1, 7, (5 << 4) | 3, 0x1b, 0x02])
    data, off = sharded.merge_bucket_records([(rec, np.array([0, len(rec)], dtype=np.uint64))] * 2, 4, 1, 2)
    assert data == rec and list(off) == [0, len(rec)]   # the same record twice merges into one
    with pytest.raises(RuntimeError):
        sharded.merge_bucket_records([(rec[:-1], np.array([0, len(rec) - 1], dtype=np.uint64))], 4, 1, 2)
    with pytest.raises(RuntimeError):
        sharded.merge_bucket_records([(rec, np.array([0, len(rec), len(rec)], dtype=np.uint64))], 4, 3, 5)
    # a fragment with one run of color-set id 2
    import struct
    frag = struct.pack("<BI", 0, 1) + struct.pack("<QI", 2, 1) + struct.pack("<I", 31) + b"A" * 31
    assert sharded.remap_frag(frag, [5, 6, 9])[5:13] == struct.pack("<Q", 9)
    with pytest.raises(RuntimeError):
        sharded.remap_frag(frag, [5, 6])
    with pytest.raises(RuntimeError):
        sharded.remap_frag(frag[:-1], [5, 6, 9])
    h, strings, soff = sharded.class_strings(np.array([0b1011], dtype=np.uint64), 4, np.array([0, 3], dtype=np.uint64))
    assert list(soff) == [0, 1, 2] and int(strings[0]) == 0b011 and int(strings[1]) == 0b1 and h[0] != h[1]
    with pytest.raises(RuntimeError):
        sharded.class_strings(np.array([0], dtype=np.uint64), 4, np.array([3, 1], dtype=np.uint64))
