"""GPU phase 1 vs the reference (golden dumps) and the oracle (fresh inputs)."""
import filecmp
import os

import pytest

from conftest import golden_case, golden_filelist
from cdbg_gpu import formats, native, synth

pytestmark = pytest.mark.gpu
CASES = ["tiny_k31", "tiny_k63", "tiny_skew_fq"]


@pytest.mark.parametrize("case", CASES)
def test_supers_match_reference_golden(engine, case, tmp_path):
    d, meta = golden_case(case)
    _, files = golden_filelist(d, tmp_path)
    hs = native.HostSequences(files)
    dump = str(tmp_path / "g.bin")
    engine.dump_supers(hs.batch, meta["k"], 0, meta["num_buckets"], dump)
    assert filecmp.cmp(dump, os.path.join(d, "supers.bin"), shallow=False)


def _fresh(tmp_path, seed, k, n=6, **kw):
    base = dict(len_min=30000, len_max=80000, div_min=0.001, div_max=0.02, indels=10, mobile_pool=3,
                mobile_min=1000, mobile_max=3000, contigs_min=1, contigs_max=20, contigs_log=1,
                lowercase_runs=1, n_runs=1)
    base.update(kw)
    p = synth.make_params(seed=seed, **base)
    return synth.write_fasta(p, n, str(tmp_path / "in"), gzip_level=1)


@pytest.mark.parametrize("k,extra", [(31, {}), (63, dict(tandem_frac=0.02, repeat_pool=3,
                                                          repeats_per_genome=4)),
                                     (31, dict(lowcomp_frac=0.10)), (21, {}), (45, {})])
def test_supers_match_oracle_fresh(engine, oracle, tmp_path, k, extra):
    lst = _fresh(tmp_path, 7 + k, k, **extra)
    files = [l.strip() for l in open(lst) if l.strip()]
    B = 512
    oracle.phase1(lst, k, B, dump=str(tmp_path / "o.bin"))
    hs = native.HostSequences(files)
    engine.dump_supers(hs.batch, k, 0, B, str(tmp_path / "g.bin"))
    assert filecmp.cmp(str(tmp_path / "o.bin"), str(tmp_path / "g.bin"), shallow=False)


@pytest.mark.parametrize("k", [31, 63])
def test_bucket_files_match_oracle(engine, oracle, tmp_path, k):
    """Canonical bucket records (full per-bucket dedup, hash order): the GPU
    bucket files decompress to exactly the oracle's record bytes."""
    lst = _fresh(tmp_path, 99 + k, k, n=8)
    files = [l.strip() for l in open(lst) if l.strip()]
    B = 256
    os.makedirs(tmp_path / "ob")
    os.makedirs(tmp_path / "gb")
    ns, nk = oracle.phase1(lst, k, B, bucket_dir=str(tmp_path / "ob"))
    st, unc = engine.phase1(files, k, B, str(tmp_path / "gb"))
    assert st.n_supers == ns and st.n_kmers == nk
    for b in range(B):
        ro = formats.read_bucket_raw(str(tmp_path / "ob" / ("bucket_%d.bin" % b)))
        rg = formats.read_bucket_raw(str(tmp_path / "gb" / ("bucket_%d.bin" % b)))
        assert ro == rg, b
        assert unc[b] == len(rg)


def test_phase1_chunked_is_valid(engine, oracle, tmp_path):
    """Several device passes (tiny chunk budget): records of a bucket are split
    across frames, the union of (bases, color) pairs per bucket is unchanged."""
    lst = _fresh(tmp_path, 5, 31, n=5)
    files = [l.strip() for l in open(lst) if l.strip()]
    B = 64
    os.makedirs(tmp_path / "a")
    os.makedirs(tmp_path / "b")
    engine.phase1(files, 31, B, str(tmp_path / "a"))
    engine.phase1(files, 31, B, str(tmp_path / "b"), chunk_bytes=1)
    for b in range(B):
        def pairs(d):
            out = set()
            for fl, cols, bases in formats.parse_records(formats.read_bucket_raw(str(d / ("bucket_%d.bin" % b)))):
                for c in cols:
                    out.add((bases, c, fl & 12))
            return out
        assert pairs(tmp_path / "a") == pairs(tmp_path / "b")


def test_sequence_boundaries_on_chunk_edges(engine, oracle, tmp_path):
    """Sequences whose starts fall on 32-byte multiples, runs that end exactly
    at a sequence end, empty sequences, N runs at the edges, lower case."""
    import random
    rnd = random.Random(5)
    seqs = []
    for i in range(60):
        n = rnd.choice([32, 64, 96, 33, 31, 128, 0, 256, 1000])
        s = "".join(rnd.choice("ACGTacgt") for _ in range(n))
        if n > 40 and i % 3 == 0:
            s = "NN" + s[2:-3] + "NNN"
        seqs.append(s)
    d = tmp_path / "in"
    os.makedirs(d)
    files = []
    for c in range(3):
        p = d / ("c%d.fa" % c)
        with open(p, "w") as f:
            for j, s in enumerate(seqs[c::3]):
                f.write(">s%d\n%s\n" % (j, s))
        files.append(str(p))
    lst = str(d / "list.txt")
    open(lst, "w").write("".join(f + "\n" for f in files))
    for k in (21, 31):
        oracle.phase1(lst, k, 64, dump=str(tmp_path / "o.bin"))
        hs = native.HostSequences(files)
        engine.dump_supers(hs.batch, k, 0, 64, str(tmp_path / "g.bin"))
        assert filecmp.cmp(str(tmp_path / "o.bin"), str(tmp_path / "g.bin"), shallow=False), k


def test_short_runs_take_the_two_pass_run_events(engine, oracle, tmp_path):
    """Sequences broken by an N every 20-40 bases: more runs than one per 64
    bases, so the one-pass run-boundary kernel's room overflows and the two
    counting passes run instead; the super-k-mers still equal the oracle's."""
    import numpy as np
    rng = np.random.default_rng(17)
    os.makedirs(tmp_path / "in")
    names = []
    for g in range(4):
        s = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=200_000)
        gaps = np.cumsum(rng.integers(20, 41, size=10_000))
        s[gaps[gaps < s.size]] = ord("N")
        path = str(tmp_path / "in" / ("g%d.fa" % g))
        with open(path, "wb") as f:
            f.write(b">g\n" + s.tobytes() + b"\n")
        names.append(path)
    lst = str(tmp_path / "in" / "filenames.txt")
    with open(lst, "w") as f:
        f.write("".join(n + "\n" for n in names))
    k, B = 21, 64
    oracle.phase1(lst, k, B, dump=str(tmp_path / "o.bin"))
    hs = native.HostSequences(names)
    engine.dump_supers(hs.batch, k, 0, B, str(tmp_path / "g.bin"))
    assert filecmp.cmp(str(tmp_path / "o.bin"), str(tmp_path / "g.bin"), shallow=False)
