"""Round 0 of the stitch on the GPU (cdbg_gpu_stitch_seed) against the
reference's own seed: the round-0 files byte for byte (LZ4 frames included)
and the closed unitigs, on the golden fragments, on synthetic fragments with
every branch of the seed, across device passes and 4 MiB frames, on a GPU
build's fragments, and through the reference's own doubling rounds and emit
to its final outputs."""
import os
import subprocess

import pytest

from conftest import golden_case, read_round_file, ref_bin, round0_files, run_ref, synth_frags
from make_golden import SEED_BUCKETS, unpack_seed

pytestmark = pytest.mark.gpu


def _seed(engine, frag, k, B, d, **kw):
    closed = os.path.join(d, "closed.bin")
    st = engine.stitch_seed(frag, k, d, num_buckets=B, closed_path=closed, **kw)
    return st, round0_files(d, B), open(closed, "rb").read()


def _ref_seed(frag, k, B, d):
    exe = ref_bin("ref_seed", k)
    if exe is None:
        pytest.skip("oracle/_ref/ref_seed not built")
    fp = os.path.join(d, "in_frag_unitigs.bin")
    os.makedirs(d, exist_ok=True)
    open(fp, "wb").write(frag)
    subprocess.run([exe, fp, str(k), str(B), "1", d], check=True, capture_output=True)
    return round0_files(d, B), open(os.path.join(d, "closed.bin"), "rb").read()


@pytest.mark.parametrize("case", ["tiny_k31", "tiny_k63", "tiny_skew_fq"])
def test_seed_equals_golden_round0_files(engine, tmp_path, case):
    d, meta = golden_case(case)
    frag = open(os.path.join(d, "frag_unitigs.bin"), "rb").read()
    st, files, closed = _seed(engine, frag, meta["k"], SEED_BUCKETS, str(tmp_path / "g"))
    assert files == unpack_seed(d)
    assert closed == open(os.path.join(d, "seed_closed.bin"), "rb").read()
    assert st["fragments"] == int(meta["phase2"]["fragments"])
    assert st["routed"] + st["closed_fragments"] == st["fragments"]


@pytest.mark.parametrize("k,B,seed", [(31, 7, 1), (63, 5, 2), (5, 3, 3), (2, 1, 4), (32, 2, 5), (47, 1024, 6)])
def test_seed_equals_reference_on_synthetic_fragments(engine, tmp_path, k, B, seed):
    frag = synth_frags(seed, 3000, k)
    ref_files, ref_closed = _ref_seed(frag, k, B, str(tmp_path / "ref"))
    st, files, closed = _seed(engine, frag, k, B, str(tmp_path / "gpu"))
    assert files == ref_files
    assert closed == ref_closed
    assert st["fragments"] == 3000


def test_seed_passes_and_frames(engine, tmp_path):
    """Many device passes (the tigs of one pass follow those of the passes
    before in every bucket) and buckets of several 4 MiB frames."""
    frag = synth_frags(9, 12000, 31, max_runs=2, max_m=3000, p_closed=0.05, p_foreign=0.0)
    for B in (1, 5):
        ref_files, ref_closed = _ref_seed(frag, 31, B, str(tmp_path / ("ref%d" % B)))
        if B == 1:
            assert len(read_round_file(os.path.join(str(tmp_path / "ref1"), "stitch_r0_b0.bin"))) >= 2
        for chunk in (0, 1 << 20, 100000):
            st, files, closed = _seed(engine, frag, 31, B, str(tmp_path / ("gpu%d_%d" % (B, chunk))),
                                      chunk_bytes=chunk)
            assert files == ref_files, (B, chunk)
            assert closed == ref_closed, (B, chunk)
            if chunk:
                assert st["n_passes"] > 1


def test_seed_closed_in_memory_and_empty_input(engine, tmp_path):
    frag = synth_frags(11, 500, 31)
    _, ref_closed = _ref_seed(frag, 31, 16, str(tmp_path / "ref"))
    st = engine.stitch_seed(frag, 31, str(tmp_path / "mem"), num_buckets=16)
    assert st["closed"] == ref_closed
    st = engine.stitch_seed(b"", 31, str(tmp_path / "empty"), num_buckets=16, closed_path=str(tmp_path / "c"))
    assert st["fragments"] == 0 and round0_files(str(tmp_path / "empty"), 16) == {}
    assert open(str(tmp_path / "c"), "rb").read() == b""


def test_seed_rejects_malformed_records(engine, tmp_path):
    frag = bytearray(synth_frags(12, 50, 31, p_closed=0.0))
    with pytest.raises(RuntimeError):
        engine.stitch_seed(bytes(frag[:-3]), 31, str(tmp_path / "a"), num_buckets=4)   # truncated
    bad = bytearray(frag)
    # an open fragment whose boundary k-mer holds a non-ACGT byte
    nr = int.from_bytes(bad[1:5], "little")
    s0 = 5 + 12 * nr + 4
    bad[s0] = ord("N")
    bad[s0 + int.from_bytes(bad[5 + 12 * nr:9 + 12 * nr], "little") - 1] = ord("N")
    with pytest.raises(RuntimeError):
        engine.stitch_seed(bytes(bad), 31, str(tmp_path / "b"), num_buckets=4)
    # the engine stays usable
    engine.stitch_seed(bytes(frag), 31, str(tmp_path / "c"), num_buckets=4)


@pytest.mark.parametrize("k", [31, 63])
def test_seed_of_gpu_build_equals_reference(engine, tmp_path, k):
    from cdbg_gpu import native, synth
    extra = dict(tandem_frac=0.02, repeat_pool=3, repeat_min=300, repeat_max=800) if k > 31 else {}
    p = synth.make_params(seed=40 + k, len_min=60000, len_max=120000, div_min=0.002, div_max=0.02, indels=5,
                          contigs_min=1, contigs_max=4, lowcomp_frac=0.05, **extra)
    lst = synth.write_fasta(p, 24, str(tmp_path / "in"))
    files = [l.strip() for l in open(lst) if l.strip()]
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, k, 1024, len(files))
    frag = native.result_frag_bytes(r)
    ref_files, ref_closed = _ref_seed(frag, k, 1024, str(tmp_path / "ref"))
    st, files_, closed = _seed(engine, frag, k, 1024, str(tmp_path / "gpu"))
    assert st["fragments"] == r.n_fragments
    assert files_ == ref_files
    assert closed == ref_closed


@pytest.mark.parametrize("k", [31, 63])
def test_gpu_seed_then_reference_rounds_equal_reference_build(engine, tmp_path, k):
    """The reference's complete build (-t 1) and its phase 2 on its own bucket
    files give a frag file; round 0 seeded from it on the GPU, then the
    reference's own doubling rounds and emit (ref_phase34 with the seed's
    outputs), reproduce the complete build's outputs byte for byte."""
    from cdbg_gpu import formats, synth
    cdbg, r2, r34 = ref_bin("cdbg-build", k), ref_bin("ref_phase2", k), ref_bin("ref_phase34", k)
    if not (cdbg and r2 and r34):
        pytest.skip("oracle/_ref not built")
    extra = dict(tandem_frac=0.02, repeat_pool=3, repeat_min=300, repeat_max=800) if k > 31 else {}
    p = synth.make_params(seed=90 + k, len_min=20000, len_max=40000, div_min=0.002, div_max=0.02, indels=5,
                          mobile_pool=3, mobile_min=500, mobile_max=2000, contigs_min=1, contigs_max=6,
                          contigs_log=1, lowcomp_frac=0.05, **extra)
    lst = synth.write_fasta(p, 4, str(tmp_path / "in"), gzip_level=1)
    ref_out = str(tmp_path / "ref" / "out")
    run_ref([cdbg, "-i", lst, "-k", str(k), "-o", ref_out, "-t", "1", "-b", "10", "-d", ref_out + "_tmp",
             "--keep-tmp"])
    run_ref([r2, ref_out + "_tmp", "1024", str(k), "4", "1", str(tmp_path / "p2")])
    _, _, _, classes = formats.read_color_sets(str(tmp_path / "p2" / "out.color_sets"))
    os.makedirs(tmp_path / "mine")
    out = str(tmp_path / "mine" / "out")
    formats.write_classes(out + ".classes", classes)
    frag_path = str(tmp_path / "p2" / "frag_unitigs.bin")
    closed = str(tmp_path / "mine" / "closed.bin")
    engine.stitch_seed(open(frag_path, "rb").read(), k, out + "_tmp", num_buckets=1024, closed_path=closed)
    run_ref([r34, frag_path, out + ".classes", "4", str(k), "1", out, out + "_tmp", closed])
    for ext in (".fa", ".color_sets", ".metadata.txt", ".u2c"):
        assert open(out + ext, "rb").read() == open(ref_out + ext, "rb").read(), ext


@pytest.mark.parametrize("k", [31, 63])
def test_build_files_seeds_round0_from_hbm(engine, tmp_path, k):
    """cdbg_gpu_build_files with stitch_dir: round 0 seeded from the fragments
    in HBM equals the reference's seed of the frag file the same call writes,
    and the same without writing the frag file at all."""
    from cdbg_gpu import formats, synth
    extra = dict(tandem_frac=0.02, repeat_pool=3, repeat_min=300, repeat_max=800) if k > 31 else {}
    p = synth.make_params(seed=70 + k, len_min=50000, len_max=90000, div_min=0.002, div_max=0.02, indels=5,
                          contigs_min=1, contigs_max=4, lowcomp_frac=0.05, **extra)
    lst = synth.write_fasta(p, 12, str(tmp_path / "in"), gzip_level=1)
    files = [l.strip() for l in open(lst) if l.strip()]
    fp, cs = str(tmp_path / "frag_unitigs.bin"), str(tmp_path / "out.color_sets")
    d1 = str(tmp_path / "r1")
    r = engine.build_files(files, k, 512, frag_path=fp, color_sets_path=cs, stitch_dir=d1, stitch_buckets=64)
    frag = open(fp, "rb").read()
    assert len(frag) == r.frag_nbytes and r.seed_routed > 0
    ref_files, ref_closed = _ref_seed(frag, k, 64, str(tmp_path / "ref"))
    assert round0_files(d1, 64) == ref_files
    assert open(os.path.join(d1, "stitch_r0_closed.bin"), "rb").read() == ref_closed
    # no frag file, no color-set file: the classes come back in host memory
    d2 = str(tmp_path / "r2")
    r2 = engine.build_files(files, k, 512, stitch_dir=d2, stitch_buckets=64,
                            stitch_closed_path=str(tmp_path / "closed2.bin"))
    assert round0_files(d2, 64) == ref_files
    assert open(str(tmp_path / "closed2.bin"), "rb").read() == ref_closed
    assert not r2.frag_bytes and r2.frag_nbytes == r.frag_nbytes
    from cdbg_gpu import native
    classes = formats.decode_classes(native.result_class_words(r2), native.result_class_offsets(r2), len(files))
    _, _, _, ref_classes = formats.read_color_sets(cs)
    assert classes == ref_classes
