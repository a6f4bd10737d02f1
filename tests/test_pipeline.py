"""Whole pipeline: phase-1 + phase-2 artifacts from this project drive the
reference's own, unchanged phase 3 (stitch) and phase 4 (emit), and the final
outputs equal those of the reference's complete cdbg-build on the same inputs.

Final outputs are compared as the multiset of (canonical unitig, decoded color
set) pairs, the color-set family and every metadata count: the reference's
bucket files depend on thread interleaving and its color-set ids on bucket
scheduling, so ids and unitig order are not comparable, the content is.

The CPU test runs the oracle's phases 1 + 2; the GPU test runs this
project's kernels (bucket files on disk, then the in-memory build)."""
import os
import subprocess

import pytest

from conftest import ref_bin, run_ref
from cdbg_gpu import formats, synth


def _inputs(tmp_path, seed, k, n=6):
    extra = dict(tandem_frac=0.02, repeat_pool=3, repeat_min=300, repeat_max=800) if k > 31 else {}
    p = synth.make_params(seed=seed, len_min=20000, len_max=40000, div_min=0.002, div_max=0.02, indels=5,
                          mobile_pool=3, mobile_min=500, mobile_max=2000, contigs_min=1, contigs_max=6,
                          contigs_log=1, lowcomp_frac=0.05, lowercase_runs=1, n_runs=1, **extra)
    return synth.write_fasta(p, n, str(tmp_path / "in"), gzip_level=1)


def _reference_build(lst, k, blog2, out, threads=2):
    cdbg = ref_bin("cdbg-build", k)
    run_ref([cdbg, "-i", lst, "-k", str(k), "-o", out, "-t", str(threads), "-b", str(blog2), "-d",
             out + "_tmp"])
    return formats.final_pairs(out, k)


def _phase34(frag, classes, C, k, out):
    cl = out + ".classes"
    formats.write_classes(cl, classes)
    run_ref([ref_bin("ref_phase34", k), frag, cl, str(C), str(k), "2", out, out + "_tmp"])
    return formats.final_pairs(out, k)


def _same(a, b):
    pa, ma, fa = a
    pb, mb, fb = b
    assert ma == mb
    assert fa == fb
    assert pa == pb


def _needs_ref(k):
    if not (ref_bin("cdbg-build", k) and ref_bin("ref_phase34", k)):
        pytest.skip("oracle/_ref not built")


@pytest.mark.parametrize("k", [31, 63])
def test_oracle_phases_drive_reference_stitch_and_emit(oracle, tmp_path, k):
    _needs_ref(k)
    lst = _inputs(tmp_path, 300 + k, k)
    n, blog2 = 6, 10
    ref = _reference_build(lst, k, blog2, str(tmp_path / "ref" / "out"))
    bdir = str(tmp_path / "b")
    os.makedirs(bdir)
    oracle.phase1(lst, k, 1 << blog2, bucket_dir=bdir)
    oracle.phase2(bdir, 1 << blog2, k, n, str(tmp_path / "o2"))
    _, _, _, classes = formats.read_color_sets(str(tmp_path / "o2" / "out.color_sets"))
    os.makedirs(tmp_path / "mine")
    got = _phase34(str(tmp_path / "o2" / "frag_unitigs.bin"), classes, n, k, str(tmp_path / "mine" / "out"))
    _same(got, ref)


def test_phase34_runner_matches_reference_on_reference_buckets(tmp_path):
    """The runner itself: the reference's own phase 2 output fed through it
    reproduces the reference's complete build byte for byte (-t 1)."""
    k = 31
    _needs_ref(k)
    r2 = ref_bin("ref_phase2", k)
    lst = _inputs(tmp_path, 77, k, n=4)
    ref_out = str(tmp_path / "ref" / "out")
    cdbg = ref_bin("cdbg-build", k)
    run_ref([cdbg, "-i", lst, "-k", str(k), "-o", ref_out, "-t", "1", "-b", "10", "-d", ref_out + "_tmp",
             "--keep-tmp"])
    bdir = ref_out + "_tmp"
    run_ref([r2, bdir, "1024", str(k), "4", "1", str(tmp_path / "p2")])
    _, _, _, classes = formats.read_color_sets(str(tmp_path / "p2" / "out.color_sets"))
    os.makedirs(tmp_path / "mine")
    out = str(tmp_path / "mine" / "out")
    formats.write_classes(out + ".classes", classes)
    run_ref([ref_bin("ref_phase34", k), str(tmp_path / "p2" / "frag_unitigs.bin"), out + ".classes", "4",
             str(k), "1", out, out + "_tmp"])
    for ext in (".fa", ".color_sets", ".metadata.txt", ".u2c"):
        assert open(out + ext, "rb").read() == open(ref_out + ext, "rb").read(), ext


@pytest.mark.gpu
@pytest.mark.parametrize("k", [31, 63])
def test_gpu_phases_drive_reference_stitch_and_emit(engine, tmp_path, k):
    _needs_ref(k)
    from cdbg_gpu import native
    lst = _inputs(tmp_path, 500 + k, k)
    n, blog2 = 6, 10
    B = 1 << blog2
    ref = _reference_build(lst, k, blog2, str(tmp_path / "ref" / "out"))
    files = [l.strip() for l in open(lst) if l.strip()]
    # bucket files on disk, then phase 2 from them
    bdir = str(tmp_path / "gb")
    os.makedirs(bdir)
    engine.phase1(files, k, B, bdir)
    frag = str(tmp_path / "frag_unitigs.bin")
    classes = []
    engine.phase2(bdir, B, k, n, frag, None, on_class=lambda c: classes.append(list(c)))
    os.makedirs(tmp_path / "mine")
    _same(_phase34(frag, classes, n, k, str(tmp_path / "mine" / "out")), ref)
    # in-memory build (no bucket files)
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, k, B, n)
    frag2 = str(tmp_path / "frag_mem.bin")
    with open(frag2, "wb") as f:
        f.write(native.result_frag_bytes(r))
    classes2 = formats.decode_classes(native.result_class_words(r), native.result_class_offsets(r), n)
    os.makedirs(tmp_path / "mem")
    _same(_phase34(frag2, classes2, n, k, str(tmp_path / "mem" / "out")), ref)


@pytest.mark.gpu
def test_gpu_pipeline_small_config_equals_reference(engine, tmp_path):
    """The small benchmark configuration at full size (10 genomes of ~5.0 Mbp,
    0.5% SNPs, 20 indels, mobile inserts, 1-3 contigs; k=31, -b 10): GPU phases
    1 + 2 through the reference's phases 3 + 4 equal the reference's own
    complete build (-t 1)."""
    k = 31
    _needs_ref(k)
    p, n, k2, blog2 = synth.preset("small", seed=5)
    assert (n, k2, blog2) == (10, 31, 10)
    lst = synth.write_fasta(p, n, str(tmp_path / "in"))
    ref = _reference_build(lst, k, blog2, str(tmp_path / "ref" / "out"), threads=1)
    files = [l.strip() for l in open(lst) if l.strip()]
    bdir = str(tmp_path / "gb")
    os.makedirs(bdir)
    engine.phase1(files, k, 1 << blog2, bdir)
    frag = str(tmp_path / "frag_unitigs.bin")
    classes = []
    engine.phase2(bdir, 1 << blog2, k, n, frag, None, on_class=lambda c: classes.append(list(c)))
    os.makedirs(tmp_path / "mine")
    _same(_phase34(frag, classes, n, k, str(tmp_path / "mine" / "out")), ref)
