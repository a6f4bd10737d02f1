"""GPU: the end-to-end in-memory build from files (cdbg_gpu_build_files):
gzip/plain FASTA or FASTQ files in, frag_unitigs.bin and a finalized
.color_sets out.  Its files must equal the drop-in path's (cdbg_gpu_phase1 +
cdbg_gpu_phase2, which the phase-2 tests pin to the reference's own
process_buckets byte for byte): the frag file byte for byte, and the
.color_sets file -- whose Elias-Fano finalize (streaming_color_set_dict.hpp:
221-294) runs on the device here and on the host there -- byte for byte."""
import filecmp
import gzip
import os
import shutil

import pytest

from cdbg_gpu import native, synth

pytestmark = pytest.mark.gpu


def _inputs(tmp_path, n, gz, seed=31, **kw):
    base = dict(len_min=40000, len_max=120000, div_min=0.001, div_max=0.02, indels=10, mobile_pool=3,
                mobile_min=1000, mobile_max=3000, contigs_min=1, contigs_max=20, contigs_log=1,
                lowercase_runs=1, n_runs=1)
    base.update(kw)
    p = synth.make_params(seed=seed, **base)
    lst = synth.write_fasta(p, n, str(tmp_path / "in"), gzip_level=1 if gz else 0)
    return [l.strip() for l in open(lst) if l.strip()]


def _dropin(engine, tmp_path, files, k, B):
    bd = tmp_path / "buckets"
    os.makedirs(bd)
    engine.phase1(files, k, B, str(bd))
    frag, cs = str(tmp_path / "want.frag"), str(tmp_path / "want.color_sets")
    engine.phase2(str(bd), B, k, len(files), frag, cs)
    return frag, cs


@pytest.mark.parametrize("k,gz,n", [(31, True, 12), (63, False, 6)])
def test_build_files_equals_dropin(engine, tmp_path, k, gz, n):
    files = _inputs(tmp_path, n, gz, tandem_frac=0.01 if k > 31 else 0.0)
    B = 256
    want_frag, want_cs = _dropin(engine, tmp_path, files, k, B)
    frag, cs = str(tmp_path / "frag_unitigs.bin"), str(tmp_path / "out.color_sets")
    for _ in range(2):  # twice: the engine's buffers are reused
        r = engine.build_files(files, k, B, frag, cs, host_threads=4)
        assert filecmp.cmp(frag, want_frag, shallow=False)
        assert filecmp.cmp(cs, want_cs, shallow=False)
    assert r.n_kmers > 0 and r.frag_nbytes == os.path.getsize(frag)
    # outputs kept in host memory instead of files
    rh = engine.build_files(files, k, B)
    assert native.result_frag_bytes(rh) == open(want_frag, "rb").read()
    # outputs on a RAM-backed file system (filled through a shared mapping)
    if os.path.isdir("/dev/shm") and os.access("/dev/shm", os.W_OK):
        import tempfile
        d = tempfile.mkdtemp(prefix="cdbg_test_", dir="/dev/shm")
        try:
            frag2, cs2 = os.path.join(d, "frag_unitigs.bin"), os.path.join(d, "out.color_sets")
            engine.build_files(files, k, B, frag2, cs2, host_threads=4)
            assert filecmp.cmp(frag2, want_frag, shallow=False)
            assert filecmp.cmp(cs2, want_cs, shallow=False)
        finally:
            shutil.rmtree(d, ignore_errors=True)


def test_multi_member_gzip_falls_back_to_whole_read(engine, tmp_path):
    """A gzip file of two members: its size field covers the last member only,
    so the streamed reader's buffers are too small; the call still gives the
    same files (it reads everything first instead)."""
    files = _inputs(tmp_path, 5, False, seed=44)
    raw = open(files[2], "rb").read()
    half = len(raw) // 2
    cut = raw.index(b">", half) if b">" in raw[half:] else len(raw)
    mm = str(tmp_path / "in" / "multi.fa.gz")
    with open(mm, "wb") as f:
        f.write(gzip.compress(raw[:cut]))
        f.write(gzip.compress(raw[cut:]))
    files[2] = mm
    B = 128
    want_frag, want_cs = _dropin(engine, tmp_path, files, 31, B)
    frag, cs = str(tmp_path / "f.bin"), str(tmp_path / "c.color_sets")
    engine.build_files(files, 31, B, frag, cs)
    assert filecmp.cmp(frag, want_frag, shallow=False)
    assert filecmp.cmp(cs, want_cs, shallow=False)


def test_fastq_and_empty_inputs(engine, tmp_path):
    """FASTQ files and a file with no sequence at all (a color without
    k-mers) go through both paths alike."""
    import make_golden
    files = _inputs(tmp_path, 4, False, seed=55)
    fq = []
    for i, f in enumerate(files):
        out = str(tmp_path / ("g%d.fq" % i))
        make_golden.to_fastq(f, out)
        fq.append(out)
    empty = str(tmp_path / "empty.fa")
    open(empty, "w").write(">nothing\n\n")
    fq.insert(1, empty)
    want_frag, want_cs = _dropin(engine, tmp_path, fq, 31, 64)
    frag, cs = str(tmp_path / "f.bin"), str(tmp_path / "c.color_sets")
    engine.build_files(fq, 31, 64, frag, cs)
    assert filecmp.cmp(frag, want_frag, shallow=False)
    assert filecmp.cmp(cs, want_cs, shallow=False)
