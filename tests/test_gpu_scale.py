"""GPU parity at the shapes the benchmarks run, against the reference itself.

Each case generates a cut of one benchmark workload with that workload's own
generator parameters (fewer genomes and shorter genomes so that the
reference's single-thread phase 2 finishes in well under a minute), then:

* GPU phase 1 writes bucket files that decompress to exactly the oracle's
  canonical records (bucket_ingester.hpp:36-177 + bucket_io.hpp:127-277);
* the reference's own process_buckets (oracle/_ref/ref_phase2, one thread,
  bucket_walker.hpp:607-779) runs on those bucket files;
* the GPU path the bench times end to end (cdbg_gpu_build_files: phases 1 +
  2 in HBM from the gzip files, no bucket files), the same build from host
  sequences (cdbg_gpu_build) and the drop-in file path (cdbg_gpu_phase2) must
  all give frag_unitigs.bin and .color_sets byte-identical to the reference's.

The shapes are asserted too, so each case really exercises what its workload
stresses: color sets hundreds of colors wide and records of >= 64 colors
(the heavy-bitmap unions) for the pangenome cut, k = 63 with 128-bit k-mers
and branching repeats for the large-k cut, and a max/median of k-mer
occurrences per bucket above 100 for the skewed cut.
"""
import filecmp
import os

import numpy as np
import pytest

from conftest import ref_bin, run_ref
from cdbg_gpu import formats, native, synth

pytestmark = pytest.mark.gpu

# name -> (preset, genomes, genome-length scale, parameter overrides)
CASES = {
    # 128 genomes of ~0.96 Mbp, 0.1-2% SNPs, 1-200 contigs: k=31, 4096 buckets
    "pangenome128": ("pangenome", 128, 0.2, {}),
    # 50 genomes of ~1.44 Mbp + 2% tandem repeats + 200 shared 1-5 kbp repeats
    # each: k=63 (128-bit k-mers), 4096 buckets
    "largek50": ("largek", 50, 0.3, {}),
    # 100 genomes of 0.5-3 Mbp log-uniform with 10% homopolymer/dinucleotide
    # runs: k=31, 16384 buckets
    "skewed100": ("skewed", 100, 0.5, {}),
}


def _same_bucket_files(gb, ob, B):
    """Bucket files equal as files, or else as decompressed record bytes."""
    for b in range(B):
        g, o = str(gb / ("bucket_%d.bin" % b)), str(ob / ("bucket_%d.bin" % b))
        if not filecmp.cmp(g, o, shallow=False):
            assert formats.read_bucket_raw(g) == formats.read_bucket_raw(o), b


def _run_case(engine, oracle, tmp_path, name):
    r2 = ref_bin("ref_phase2", 63 if name.startswith("largek") else 31)
    if not r2:
        pytest.skip("oracle/_ref not built")
    pre, n, scale, ov = CASES[name]
    p, _, k, blog = synth.preset(pre, seed=7, scale=scale, **ov)
    B = 1 << blog
    lst = synth.write_fasta(p, n, str(tmp_path / "in"), gzip_level=1)
    files = [l.strip() for l in open(lst) if l.strip()]
    gb, ob = tmp_path / "gb", tmp_path / "ob"
    os.makedirs(gb)
    os.makedirs(ob)

    # phase 1: GPU bucket files == the oracle's canonical records
    st, unc = engine.phase1(files, k, B, str(gb))
    ns, nk = oracle.phase1(lst, k, B, bucket_dir=str(ob))
    assert (st.n_supers, st.n_kmers) == (ns, nk)
    _same_bucket_files(gb, ob, B)

    # the reference's own phase 2, one thread (deterministic ids and order)
    run_ref([r2, str(gb), str(B), str(k), str(n), "1", str(tmp_path / "ref")])
    ref_frag_p = str(tmp_path / "ref" / "frag_unitigs.bin")
    ref_cs_p = str(tmp_path / "ref" / "out.color_sets")

    # the drop-in file path
    frag = str(tmp_path / "frag_unitigs.bin")
    cs = str(tmp_path / "out.color_sets")
    engine.phase2(str(gb), B, k, n, frag, cs)
    assert filecmp.cmp(frag, ref_frag_p, shallow=False)
    assert filecmp.cmp(cs, ref_cs_p, shallow=False)

    # the benchmarked path, end to end from the files (phases 1 + 2 in HBM)
    engine.build_files(files, k, B, frag, cs)
    assert filecmp.cmp(frag, ref_frag_p, shallow=False)
    assert filecmp.cmp(cs, ref_cs_p, shallow=False)

    # and from host sequences, outputs in host memory
    C, ref_words, ref_offs, _ = formats.read_color_sets(ref_cs_p, decode=False)
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, k, B, n)
    assert r.n_kmers == nk
    assert native.result_frag_bytes(r) == open(ref_frag_p, "rb").read()
    assert list(native.result_class_offsets(r)) == list(ref_offs)
    assert np.array_equal(native.result_class_words(r), ref_words)
    return dict(k=k, B=B, lst=lst, words=ref_words, offs=ref_offs, nbits=int(r.class_bits), gb=gb, n=n)


def _class_sizes(c, count=4000):
    """Color counts of a random sample of the classes (the size leads each
    class's encoding)."""
    w = np.append(c["words"], np.uint64(0))
    offs = c["offs"]
    idx = np.random.default_rng(0).choice(len(offs), size=min(count, len(offs)), replace=False)
    return [formats.read_delta(formats._Bits(w, int(offs[i]))) for i in idx]


def test_pangenome_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "pangenome128")
    assert max(_class_sizes(c)) >= 100                # classes a hundred colors wide and more
    heavy = 0
    for b in range(0, c["B"], 256):                   # records of >= 64 colors exist
        for _, cols, _ in formats.parse_records(formats.read_bucket_raw(str(c["gb"] / ("bucket_%d.bin" % b)))):
            heavy += len(cols) >= 64
    assert heavy > 0


def test_largek_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "largek50")
    assert c["k"] == 63
    assert len(c["offs"]) > 1000


def test_skewed_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "skewed100")
    # heavy-tailed buckets: k-mer occurrences per bucket before deduplication
    occ = oracle.bucket_kmers(c["lst"], c["k"], c["B"]).astype(np.float64)
    med = float(np.median(occ[occ > 0]))
    assert occ.max() / med > 100, (occ.max(), med)
