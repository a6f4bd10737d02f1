"""GPU phase 2 vs the reference's own process_buckets (golden outputs and
oracle/_ref runs): frag_unitigs.bin and .color_sets must be byte-identical."""
import filecmp
import os
import shutil

import numpy as np
import pytest

from conftest import golden_case, golden_filelist, ref_bin, run_ref
from cdbg_gpu import formats, native, synth
import make_golden

pytestmark = pytest.mark.gpu
CASES = ["tiny_k31", "tiny_k63", "tiny_skew_fq"]


@pytest.mark.parametrize("case", CASES)
def test_phase2_on_reference_buckets(engine, case, tmp_path):
    d, meta = golden_case(case)
    bdir = str(tmp_path / "b")
    make_golden.unpack_buckets(d, bdir)
    frag = str(tmp_path / "frag_unitigs.bin")
    cs = str(tmp_path / "out.color_sets")
    st = engine.phase2(bdir, meta["num_buckets"], meta["k"], meta["num_colors"], frag, cs)
    assert st.n_fragments == int(meta["phase2"]["fragments"])
    assert st.n_color_sets == int(meta["phase2"]["num_color_sets"])
    assert filecmp.cmp(frag, os.path.join(d, "frag_unitigs.bin"), shallow=False)
    assert filecmp.cmp(cs, os.path.join(d, "out.color_sets"), shallow=False)


def _fresh(tmp_path, seed, n, **kw):
    base = dict(len_min=40000, len_max=90000, div_min=0.001, div_max=0.02, indels=10, mobile_pool=3,
                mobile_min=1000, mobile_max=3000, contigs_min=1, contigs_max=20, contigs_log=1,
                lowercase_runs=1, n_runs=1)
    base.update(kw)
    p = synth.make_params(seed=seed, **base)
    return synth.write_fasta(p, n, str(tmp_path / "in"))


@pytest.mark.parametrize("k,n,B,extra", [
    (31, 8, 128, {}),
    (63, 6, 128, dict(tandem_frac=0.02, repeat_pool=4, repeats_per_genome=6)),
    (31, 10, 64, dict(lowcomp_frac=0.10)),
    (31, 40, 256, dict(len_min=10000, len_max=30000)),
])
def test_phase2_vs_reference_fresh(engine, oracle, tmp_path, k, n, B, extra):
    r2 = ref_bin("ref_phase2", k)
    if not r2:
        pytest.skip("oracle/_ref not built")
    lst = _fresh(tmp_path, 1000 + k + n, n, **extra)
    files = [l.strip() for l in open(lst) if l.strip()]
    bdir = tmp_path / "gb"
    os.makedirs(bdir)
    engine.phase1(files, k, B, str(bdir))
    run_ref([r2, str(bdir), str(B), str(k), str(n), "1", str(tmp_path / "ref")])
    frag = str(tmp_path / "frag_unitigs.bin")
    cs = str(tmp_path / "out.color_sets")
    engine.phase2(str(bdir), B, k, n, frag, cs)
    assert filecmp.cmp(frag, str(tmp_path / "ref" / "frag_unitigs.bin"), shallow=False)
    assert filecmp.cmp(cs, str(tmp_path / "ref" / "out.color_sets"), shallow=False)


def test_batching_does_not_change_results(engine, tmp_path):
    lst = _fresh(tmp_path, 77, 6)
    files = [l.strip() for l in open(lst) if l.strip()]
    B = 128
    bdir = tmp_path / "gb"
    os.makedirs(bdir)
    engine.phase1(files, 31, B, str(bdir))
    outs = []
    for occ in (0, 5000, 100000):
        frag = str(tmp_path / ("f%d" % occ))
        cs = str(tmp_path / ("c%d" % occ))
        engine.phase2(str(bdir), B, 31, 6, frag, cs, batch_occ=occ)
        outs.append((open(frag, "rb").read(), open(cs, "rb").read()))
    assert outs[0] == outs[1] == outs[2]


def test_in_memory_build_matches_file_path(engine, tmp_path):
    lst = _fresh(tmp_path, 5, 5)
    files = [l.strip() for l in open(lst) if l.strip()]
    B, k = 128, 31
    bdir = tmp_path / "gb"
    os.makedirs(bdir)
    engine.phase1(files, k, B, str(bdir))
    frag = str(tmp_path / "frag")
    classes = []
    engine.phase2(str(bdir), B, k, 5, frag, str(tmp_path / "cs"), on_class=lambda c: classes.append(list(c)))
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, k, B, 5)
    assert native.result_frag_bytes(r) == open(frag, "rb").read()
    C, words, offsets, decoded = formats.read_color_sets(str(tmp_path / "cs"))
    assert list(native.result_class_offsets(r)) == offsets
    assert np.array_equal(native.result_class_words(r), words)
    assert decoded == classes


def test_device_resident_outputs_match_host_outputs(engine, tmp_path):
    """cdbg_gpu_build with outputs left in HBM returns the same bytes."""
    lst = _fresh(tmp_path, 21, 5)
    files = [l.strip() for l in open(lst) if l.strip()]
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, 31, 128, 5)
    frag, words = native.result_frag_bytes(r), native.result_class_words(r).tobytes()
    offs = native.result_class_offsets(r).tobytes()
    for _ in range(2):  # twice: outputs are reused buffers
        rd = engine.build(hs.batch, 31, 128, 5, outputs_to_host=False)
        assert rd.frag_nbytes == len(frag) and rd.n_color_sets == r.n_color_sets
        assert engine.copy_out(rd.frag_bytes, rd.frag_nbytes) == frag
        assert engine.copy_out(rd.class_words, len(words)) == words
        assert engine.copy_out(rd.class_offsets, len(offs)) == offs


def test_union_list_path_matches_bitmap_path(engine, tmp_path):
    """Multi-record color unions as lists (used above 8192 colors) give the
    same bytes as the bitmap path."""
    lst = _fresh(tmp_path, 31, 8)
    files = [l.strip() for l in open(lst) if l.strip()]
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, 31, 128, 8)
    a = (native.result_frag_bytes(r), native.result_class_words(r).tobytes())
    engine.set_tuning(union_lists=1)
    try:
        r2 = engine.build(hs.batch, 31, 128, 8)
    finally:
        engine.set_tuning()
    assert (native.result_frag_bytes(r2), native.result_class_words(r2).tobytes()) == a


def test_streamed_host_outputs_match_across_build_sizes(tmp_path):
    """Host outputs of in-memory builds, whose fragment bytes, class words
    and class offsets go to pinned memory batch by batch while later batches
    run once the engine's buffers are large enough (else in one copy at the
    end): identical whatever the order of build sizes and bucket-batch sizes."""
    small = native.HostSequences([l.strip() for l in open(_fresh(tmp_path / "s", 61, 3)) if l.strip()])
    large = native.HostSequences([l.strip() for l in open(_fresh(tmp_path / "l", 62, 12)) if l.strip()])
    B, k = 256, 31

    def outs(e, hs, n, batch_occ=0):
        r = e.build(hs.batch, k, B, n, batch_occ=batch_occ)
        return (native.result_frag_bytes(r), native.result_class_words(r).tobytes(),
                native.result_class_offsets(r).tobytes())

    ref = native.Engine(0)
    want_s, want_l = outs(ref, small, 3), outs(ref, large, 12)
    ref.close()
    e = native.Engine(0)
    try:
        assert outs(e, small, 3) == want_s          # nothing pinned yet: one copy at the end
        assert outs(e, large, 12, 1 << 12) == want_l  # larger than the buffer: falls back
        assert outs(e, large, 12, 1 << 12) == want_l  # streamed, many batches
        assert outs(e, small, 3, 1 << 10) == want_s   # streamed into the larger buffer
    finally:
        e.close()


def test_pipelined_host_upload_matches_device_input():
    """Host inputs of 64 MB and more are uploaded in pieces while phase 1
    works on the pieces already on the device; the outputs equal those of
    the same sequences given already in device memory (one pass)."""
    import torch
    p, _, k, blog2 = synth.preset("small", seed=9)
    n = 16
    seq, lens, per = synth.collection(p, n)
    assert seq.nbytes >= (64 << 20)
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    colors = np.repeat(np.arange(n, dtype=np.uint32), per)
    e = native.Engine(0)
    try:
        r = e.build(native.array_batch(seq, off, colors), k, 1 << blog2, n)
        host = (native.result_frag_bytes(r), native.result_class_words(r), native.result_class_offsets(r),
                r.n_kmers, r.n_supers, r.n_records)
        d_seq = torch.from_numpy(seq).cuda()
        d_off = torch.from_numpy(off.view(np.int64)).cuda()
        d_col = torch.from_numpy(colors.view(np.int32)).cuda()
        torch.cuda.synchronize()
        b = native.SeqBatch(d_seq.data_ptr(), seq.nbytes, d_off.data_ptr(), d_col.data_ptr(), len(colors), 1)
        r2 = e.build(b, k, 1 << blog2, n)
        dev = (native.result_frag_bytes(r2), native.result_class_words(r2), native.result_class_offsets(r2),
               r2.n_kmers, r2.n_supers, r2.n_records)
    finally:
        e.close()
    assert host[0] == dev[0]
    assert np.array_equal(host[1], dev[1]) and np.array_equal(host[2], dev[2])
    assert host[3:] == dev[3:]


def test_phase2_range_by_range_matches_one_pass(engine, tmp_path):
    """The drop-in phase 2 reads buckets range by range (the class
    dictionary continues across ranges); with ranges of a few buckets each,
    or a memory cap below the total bucket bytes, the frag file and
    .color_sets equal the one-pass result and the reference's own
    process_buckets, and delete_consumed leaves no bucket file behind."""
    r2 = ref_bin("ref_phase2", 31)
    lst = _fresh(tmp_path, 311, 12)
    files = [l.strip() for l in open(lst) if l.strip()]
    B, k = 128, 31
    bdir = tmp_path / "gb"
    os.makedirs(bdir)
    _, unc = engine.phase1(files, k, B, str(bdir))
    total = int(unc.sum())
    one = (str(tmp_path / "f1"), str(tmp_path / "c1"))
    s1 = engine.phase2(str(bdir), B, k, 12, *one, pass_bytes=total * 2)
    assert s1.n_passes == 1
    many = (str(tmp_path / "f2"), str(tmp_path / "c2"))
    s2 = engine.phase2(str(bdir), B, k, 12, *many, pass_bytes=max(1, total // 9))
    assert s2.n_passes >= 9
    for a, b in zip(one, many):
        assert filecmp.cmp(a, b, shallow=False)
    if r2:
        run_ref([r2, str(bdir), str(B), str(k), "12", "1", str(tmp_path / "ref")])
        assert filecmp.cmp(one[0], str(tmp_path / "ref" / "frag_unitigs.bin"), shallow=False)
        assert filecmp.cmp(one[1], str(tmp_path / "ref" / "out.color_sets"), shallow=False)
    # a memory cap below the bucket bytes: automatic ranges, same bytes, and
    # every bucket file removed once its fragments are written
    e2 = native.Engine(0)
    try:
        e2.set_memory_limit(max(total // 3, 64 << 20))
        capped = (str(tmp_path / "f3"), str(tmp_path / "c3"))
        copy = tmp_path / "gb2"
        shutil.copytree(bdir, copy)
        e2.phase2(str(copy), B, k, 12, *capped, delete_consumed=True, pass_bytes=max(1, total // 5))
        for a, b in zip(one, capped):
            assert filecmp.cmp(a, b, shallow=False)
        assert not [f for f in os.listdir(copy) if f.startswith("bucket_")]
    finally:
        e2.close()
