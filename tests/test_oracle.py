"""CPU: the oracle restatement against the reference's own outputs.

Golden fixtures (tests/golden/, made by make_golden.py from the reference
built from its sources) pin the oracle; when oracle/_ref is present the
oracle is also compared with the reference on fresh seeded inputs."""
import filecmp
import os

import pytest

from conftest import golden_case, golden_filelist, ref_bin, run_ref
import make_golden

CASES = ["tiny_k31", "tiny_k63", "tiny_skew_fq"]


@pytest.mark.parametrize("case", CASES)
def test_phase1_supers_match_reference(oracle, case, tmp_path):
    d, meta = golden_case(case)
    lst, _ = golden_filelist(d, tmp_path)
    dump = str(tmp_path / "o.bin")
    oracle.phase1(lst, meta["k"], meta["num_buckets"], dump=dump)
    assert filecmp.cmp(dump, os.path.join(d, "supers.bin"), shallow=False)


@pytest.mark.parametrize("case", CASES)
def test_phase2_matches_reference(oracle, case, tmp_path):
    d, meta = golden_case(case)
    bdir = str(tmp_path / "b")
    make_golden.unpack_buckets(d, bdir)
    out = str(tmp_path / "o")
    st = oracle.phase2(bdir, meta["num_buckets"], meta["k"], meta["num_colors"], out)
    assert st["fragments"] == int(meta["phase2"]["fragments"])
    assert st["num_color_sets"] == int(meta["phase2"]["num_color_sets"])
    assert filecmp.cmp(os.path.join(out, "frag_unitigs.bin"), os.path.join(d, "frag_unitigs.bin"),
                       shallow=False)
    assert filecmp.cmp(os.path.join(out, "out.color_sets"), os.path.join(d, "out.color_sets"),
                       shallow=False)


@pytest.mark.parametrize("k", [31, 63])
def test_oracle_vs_reference_fresh(oracle, k, tmp_path):
    """Fresh seeded input: phase-1 dumps and phase-2 outputs on the oracle's
    canonical bucket files, oracle vs the reference's own code."""
    r1, r2 = ref_bin("ref_phase1", k), ref_bin("ref_phase2", k)
    if not (r1 and r2):
        pytest.skip("oracle/_ref not built")
    from cdbg_gpu import synth
    p = synth.make_params(seed=101 + k, len_min=20000, len_max=30000, div_min=0.002, div_max=0.02,
                          indels=5, mobile_pool=3, mobile_min=500, mobile_max=2000, contigs_min=1,
                          contigs_max=5, contigs_log=1, lowcomp_frac=0.05, lowercase_runs=1, n_runs=1)
    lst = synth.write_fasta(p, 5, str(tmp_path / "in"), gzip_level=1)
    B = 128
    oracle.phase1(lst, k, B, dump=str(tmp_path / "o.bin"), bucket_dir=str(tmp_path))
    run_ref([r1, lst, str(k), "0", str(B), str(tmp_path / "r.bin")])
    assert filecmp.cmp(str(tmp_path / "o.bin"), str(tmp_path / "r.bin"), shallow=False)
    oracle.phase2(str(tmp_path), B, k, 5, str(tmp_path / "o2"))
    run_ref([r2, str(tmp_path), str(B), str(k), "5", "1", str(tmp_path / "r2")])
    for f in ("frag_unitigs.bin", "out.color_sets"):
        assert filecmp.cmp(str(tmp_path / "o2" / f), str(tmp_path / "r2" / f), shallow=False), f


def test_best_m(oracle):
    from cdbg_gpu.native import best_m
    for k in range(2, 70):
        assert oracle.L.oracle_best_m(k) == best_m(k)
