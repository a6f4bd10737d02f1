"""CPU: a build split by bucket range across ranks, merged on one rank, equals
the single build byte for byte (frag_unitigs.bin bytes, color-set bits and
offsets).

Each rank's share of the build is made here by the CPU oracle -- phase 1 of
the whole collection, then phase 2 of only the rank's bucket range, which is
what a rank's cdbg_gpu_build with that bucket range computes on its GPU (the
GPU test test_gpu_sharded.py checks that side).  What is under test is the
product's exchange and merge: cdbg_gpu/sharded.py gathering the shards over
torch.distributed (gloo, world size 2, two processes) and cdbg_merge_shards
renumbering the color sets and rewriting the fragments' ids."""
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


def _collection(d, seed=17):
    from cdbg_gpu import synth
    p = synth.make_params(seed=seed, len_min=20000, len_max=60000, div_min=0.002, div_max=0.02, indels=5,
                          mobile_pool=2, mobile_min=500, mobile_max=1500, contigs_min=1, contigs_max=8,
                          contigs_log=1, lowercase_runs=1, n_runs=1)
    return synth.write_fasta(p, N, os.path.join(d, "in"))


def _oracle_shard(orc, lst, d, lo, hi):
    """The shard of buckets [lo, hi): (frag bytes, words, bits, offsets)."""
    from cdbg_gpu import formats
    allb = os.path.join(d, "all")
    if not os.path.isdir(allb):
        os.makedirs(allb)
        orc.phase1(lst, K, B, bucket_dir=allb)
    sd = os.path.join(d, "s%d_%d" % (lo, hi))
    os.makedirs(sd)
    for b in range(lo, hi):
        src = os.path.join(allb, "bucket_%d.bin" % b)
        if os.path.exists(src):
            os.symlink(src, os.path.join(sd, "bucket_%d.bin" % b))
    out = os.path.join(sd, "out")
    orc.phase2(sd, B, K, N, out)
    frag = open(os.path.join(out, "frag_unitigs.bin"), "rb").read()
    C, words, offs, _ = formats.read_color_sets(os.path.join(out, "out.color_sets"))
    bits = int(np.fromfile(os.path.join(out, "out.color_sets"), dtype=np.uint64, count=1, offset=12)[0])
    return frag, np.asarray(words, dtype=np.uint64), bits, np.asarray(offs, dtype=np.uint64)


def _single(orc, lst, d):
    return _oracle_shard(orc, lst, d, 0, B)


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
        orc = Oracle()
        lst = os.path.join(d, "in", "filenames.txt")
        rd = os.path.join(d, "rank%d" % rank)
        os.makedirs(rd)
        lo, hi = sharded.shard_range(B, rank, world)
        shard = _oracle_shard(orc, lst, rd, lo, hi)
        merged = sharded.gather_merge(shard, rank, world)
        if rank == 0:
            frag, w, o, bits = merged
            out.put((frag, w.tobytes(), o.tobytes(), bits))
    finally:
        dist.destroy_process_group()


def test_two_ranks_merge_to_the_single_build(tmp_path):
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built")
    from conftest import Oracle
    d = str(tmp_path)
    lst = _collection(d)
    want = _single(Oracle(), lst, os.path.join(d, "single"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, d, q)) for r in range(2)]
    for p in procs:
        p.start()
    frag, w, o, bits = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert frag == want[0]
    assert w == want[1].tobytes() and bits == want[2]
    assert o == want[3].tobytes()


@pytest.mark.parametrize("world", [1, 3, 5])
def test_merge_of_any_split_is_the_single_build(tmp_path, world):
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built")
    from conftest import Oracle
    from cdbg_gpu import sharded
    orc = Oracle()
    d = str(tmp_path)
    lst = _collection(d, seed=23)
    want = _single(orc, lst, os.path.join(d, "single"))
    shards = [_oracle_shard(orc, lst, os.path.join(d, "split"), *sharded.shard_range(B, r, world))
              for r in range(world)]
    frag, w, o, bits = sharded.merge_shards(shards)
    assert frag == want[0]
    assert np.array_equal(w, want[1]) and bits == want[2]
    assert np.array_equal(o, want[3])
    # the ranks really split the color sets: some shard numbers a set
    # differently from the whole build
    if world > 1:
        assert any(len(s[3]) < len(want[3]) for s in shards)


def _intern_worker(rank, world, port, d, out):
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
        orc = Oracle()
        lst = os.path.join(d, "in", "filenames.txt")
        rd = os.path.join(d, "rank%d" % rank)
        os.makedirs(rd)
        shard = _oracle_shard(orc, lst, rd, *sharded.shard_range(B, rank, world))
        interned = sharded.intern_classes(shard, rank, world)
        whole = sharded.assemble(interned, rank, world)
        if rank == 0:
            frag, w, o, bits = whole
            out.put((frag, w.tobytes(), o.tobytes(), bits))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_hash_partitioned_interning_is_the_single_build(tmp_path, world):
    """Color sets interned across ranks (owner = class hash mod ranks, ids by a
    prefix sum over the ranks' first-seen classes, every rank rewriting its own
    fragments) equal the single build byte for byte."""
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built")
    from conftest import Oracle
    d = str(tmp_path)
    lst = _collection(d, seed=29)
    want = _single(Oracle(), lst, os.path.join(d, "single"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_intern_worker, args=(r, world, port, d, q)) for r in range(world)]
    for p in procs:
        p.start()
    frag, w, o, bits = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert frag == want[0]
    assert bits == want[2] and w == want[1].tobytes()
    assert o == want[3].tobytes()
