"""The round-0 seed restatement (oracle/stitch_seed.py) against the
reference's own seed: the golden round-0 fixtures and, where the reference
binary is built, ref_seed runs on synthetic fragments (CPU only)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT, golden_case, read_round_file, ref_bin, synth_frags

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import stitch_seed  # noqa: E402
from make_golden import SEED_BUCKETS, unpack_seed  # noqa: E402


def frames_of_bytes(data, tmp_path, name="f.bin"):
    p = os.path.join(str(tmp_path), name)
    open(p, "wb").write(data)
    return read_round_file(p)


@pytest.mark.parametrize("case", ["tiny_k31", "tiny_k63", "tiny_skew_fq"])
def test_restatement_matches_golden_seed(case, tmp_path):
    d, meta = golden_case(case)
    frag = open(os.path.join(d, "frag_unitigs.bin"), "rb").read()
    frames, closed = stitch_seed.seed(frag, meta["k"], SEED_BUCKETS)
    files = unpack_seed(d)
    assert closed == open(os.path.join(d, "seed_closed.bin"), "rb").read()
    assert sorted(files) == [b for b in range(SEED_BUCKETS) if frames[b]]
    for b, data in files.items():
        assert frames_of_bytes(data, tmp_path) == frames[b], b
    assert any(frames) and closed


@pytest.mark.parametrize("k,buckets,seed", [(31, 7, 1), (63, 5, 2), (5, 3, 3), (2, 1, 4), (32, 2, 5)])
def test_restatement_matches_ref_seed_on_synthetic_fragments(k, buckets, seed, tmp_path):
    exe = ref_bin("ref_seed", k)
    if exe is None:
        pytest.skip("oracle/_ref/ref_seed not built")
    frag = synth_frags(seed, 400, k)
    fp = os.path.join(str(tmp_path), "frag_unitigs.bin")
    open(fp, "wb").write(frag)
    out = os.path.join(str(tmp_path), "ref")
    subprocess.run([exe, fp, str(k), str(buckets), "1", out], check=True, capture_output=True)
    frames, closed = stitch_seed.seed(frag, k, buckets)
    assert closed == open(os.path.join(out, "closed.bin"), "rb").read()
    for b in range(buckets):
        p = os.path.join(out, "stitch_r0_b%d.bin" % b)
        assert os.path.exists(p) == bool(frames[b]), b
        if frames[b]:
            assert read_round_file(p) == frames[b], b


def test_restatement_frames_split_at_four_mib(tmp_path):
    """One bucket, more than 4 MiB of tigs: frames close at the first tig that
    takes the batch to 4 MiB, as round_store_file::emit flushes."""
    exe = ref_bin("ref_seed", 31)
    if exe is None:
        pytest.skip("oracle/_ref/ref_seed not built")
    frag = synth_frags(9, 12000, 31, max_runs=2, max_m=3000, p_closed=0.05, p_foreign=0.0)
    fp = os.path.join(str(tmp_path), "frag_unitigs.bin")
    open(fp, "wb").write(frag)
    out = os.path.join(str(tmp_path), "ref")
    subprocess.run([exe, fp, "31", "1", "1", out], check=True, capture_output=True)
    frames, closed = stitch_seed.seed(frag, 31, 1)
    got = read_round_file(os.path.join(out, "stitch_r0_b0.bin"))
    assert len(got) >= 2
    assert got == frames[0]
    assert closed == open(os.path.join(out, "closed.bin"), "rb").read()


@pytest.mark.parametrize("k", [31, 63])
def test_phase34_seed_mode_matches_reference_build(tmp_path, k):
    """The harness's seed mode itself: the reference's own round-0 files and
    closed unitigs (ref_seed, 1 thread) fed to ref_phase34 reproduce the
    reference's complete build (-t 1) byte for byte -- the path the GPU seed
    is checked through."""
    from cdbg_gpu import formats, synth
    cdbg, r2, r34, rs = (ref_bin(n, k) for n in ("cdbg-build", "ref_phase2", "ref_phase34", "ref_seed"))
    if not (cdbg and r2 and r34 and rs):
        pytest.skip("oracle/_ref not built")
    p = synth.make_params(seed=90 + k, len_min=20000, len_max=40000, div_min=0.002, div_max=0.02, indels=5,
                          mobile_pool=3, mobile_min=500, mobile_max=2000, contigs_min=1, contigs_max=6,
                          contigs_log=1, lowcomp_frac=0.05)
    lst = synth.write_fasta(p, 4, str(tmp_path / "in"), gzip_level=1)
    ref_out = str(tmp_path / "ref" / "out")
    subprocess.run([cdbg, "-i", lst, "-k", str(k), "-o", ref_out, "-t", "1", "-b", "10", "-d", ref_out + "_tmp",
                    "--keep-tmp"], check=True, capture_output=True)
    subprocess.run([r2, ref_out + "_tmp", "1024", str(k), "4", "1", str(tmp_path / "p2")], check=True,
                   capture_output=True)
    _, _, _, classes = formats.read_color_sets(str(tmp_path / "p2" / "out.color_sets"))
    os.makedirs(tmp_path / "mine")
    out = str(tmp_path / "mine" / "out")
    formats.write_classes(out + ".classes", classes)
    frag_path = str(tmp_path / "p2" / "frag_unitigs.bin")
    subprocess.run([rs, frag_path, str(k), "1024", "1", out + "_tmp"], check=True, capture_output=True)
    subprocess.run([r34, frag_path, out + ".classes", "4", str(k), "1", out, out + "_tmp",
                    os.path.join(out + "_tmp", "closed.bin")], check=True, capture_output=True)
    for ext in (".fa", ".color_sets", ".metadata.txt", ".u2c"):
        assert open(out + ext, "rb").read() == open(ref_out + ext, "rb").read(), ext


@pytest.mark.parametrize("threads", [1, 3, 8, 32])
def test_frag_record_offsets_parallel_scan(threads):
    """cdbg_frag_record_offsets (host threads guessing record starts in their
    share of the buffer, joined where the true records meet them) equals a
    sequential walk, with records much larger than a share among small ones."""
    import struct
    import numpy as np
    from cdbg_gpu import native
    parts = [synth_frags(21, 20000, 31, max_m=60),
             synth_frags(22, 3, 31, max_runs=1, max_m=3_000_000, p_closed=0.0),
             synth_frags(23, 20000, 63, max_m=200), synth_frags(24, 1, 31, max_runs=0, p_closed=1.0)]
    frag = b"".join(parts)
    want, p = [], 0
    while p < len(frag):
        want.append(p)
        (nr,) = struct.unpack_from("<I", frag, p + 1)
        (ln,) = struct.unpack_from("<I", frag, p + 5 + 12 * nr)
        p += 9 + 12 * nr + ln
    want.append(len(frag))
    got = native.frag_record_offsets(frag, threads)
    assert np.array_equal(got, np.array(want, dtype=np.uint64))
    with pytest.raises(RuntimeError):
        native.frag_record_offsets(frag[:-1], threads)
    assert list(native.frag_record_offsets(b"", threads)) == [0]
