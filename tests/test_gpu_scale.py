"""GPU parity at the shapes the benchmarks run, against the reference itself.

Each case generates a cut of one benchmark workload with that workload's own
generator parameters (fewer genomes and shorter genomes so that the
reference's single-thread phase 2 finishes in well under a minute), then:

* GPU phase 1 writes bucket files that decompress to exactly the oracle's
  canonical records (bucket_ingester.hpp:36-177 + bucket_io.hpp:127-277);
* the reference's own process_buckets (oracle/_ref/ref_phase2, one thread,
  bucket_walker.hpp:607-779) runs on those bucket files;
* the GPU path the bench times (cdbg_gpu_build: phases 1 + 2 in HBM, no
  bucket files) and the drop-in file path (cdbg_gpu_phase2) must both give
  frag_unitigs.bin and .color_sets byte-identical to the reference's.

The shapes are asserted too, so each case really exercises what its workload
stresses: color sets hundreds of colors wide and records of >= 64 colors
(the heavy-bitmap unions) for the pangenome cut, k = 63 with 128-bit k-mers
and branching repeats for the large-k cut, and a max/median bucket size
above 100 for the skewed cut.
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
    for b in range(B):
        rg = formats.read_bucket_raw(str(gb / ("bucket_%d.bin" % b)))
        assert rg == formats.read_bucket_raw(str(ob / ("bucket_%d.bin" % b))), b
        assert unc[b] == len(rg)

    # the reference's own phase 2, one thread (deterministic ids and order)
    run_ref([r2, str(gb), str(B), str(k), str(n), "1", str(tmp_path / "ref")])
    ref_frag = open(tmp_path / "ref" / "frag_unitigs.bin", "rb").read()
    C, ref_words, ref_offs, ref_classes = formats.read_color_sets(str(tmp_path / "ref" / "out.color_sets"))

    # the drop-in file path
    frag = str(tmp_path / "frag_unitigs.bin")
    cs = str(tmp_path / "out.color_sets")
    engine.phase2(str(gb), B, k, n, frag, cs)
    assert filecmp.cmp(frag, str(tmp_path / "ref" / "frag_unitigs.bin"), shallow=False)
    assert filecmp.cmp(cs, str(tmp_path / "ref" / "out.color_sets"), shallow=False)

    # the benchmarked path: phases 1 + 2 in HBM from host sequences
    hs = native.HostSequences(files)
    r = engine.build(hs.batch, k, B, n)
    assert r.n_kmers == nk
    assert native.result_frag_bytes(r) == ref_frag
    assert list(native.result_class_offsets(r)) == list(ref_offs)
    assert np.array_equal(native.result_class_words(r), ref_words)
    return dict(k=k, B=B, unc=unc, classes=ref_classes, gb=gb, n=n)


def test_pangenome_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "pangenome128")
    widths = [len(x) for x in c["classes"]]
    assert max(widths) >= 100, max(widths)          # classes hundreds of colors wide
    heavy = 0
    for b in range(0, c["B"], 16):                  # records of >= 64 colors exist
        for _, cols, _ in formats.parse_records(formats.read_bucket_raw(str(c["gb"] / ("bucket_%d.bin" % b)))):
            heavy += len(cols) >= 64
    assert heavy > 0


def test_largek_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "largek50")
    assert c["k"] == 63
    assert len(c["classes"]) > 1000


def test_skewed_cut_matches_reference(engine, oracle, tmp_path):
    c = _run_case(engine, oracle, tmp_path, "skewed100")
    unc = np.asarray(c["unc"], dtype=np.float64)
    med = float(np.median(unc[unc > 0]))
    assert unc.max() / med > 100, (unc.max(), med)  # heavy-tailed buckets
