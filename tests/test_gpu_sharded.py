"""GPU: a build split by bucket range (cdbg_gpu_build with bucket_lo/hi, one
call per rank's share, here one after another on one GPU) merged with
cdbg_merge_shards equals the single build byte for byte: the frag bytes, the
color-set bit vector and its offsets.  The exchange between ranks is covered
on CPU by test_sharded.py."""
import numpy as np
import pytest

from cdbg_gpu import native, sharded, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k,world", [(31, 2), (31, 3), (63, 2)])
def test_split_build_merges_to_single(engine, tmp_path, k, world):
    p = synth.make_params(seed=40 + k + world, len_min=30000, len_max=90000, div_min=0.001, div_max=0.02,
                          indels=8, mobile_pool=3, mobile_min=800, mobile_max=2000, contigs_min=1,
                          contigs_max=12, contigs_log=1, lowercase_runs=1, n_runs=1,
                          tandem_frac=0.01 if k > 31 else 0.0)
    n, B = 10, 256
    lst = synth.write_fasta(p, n, str(tmp_path / "in"))
    hs = native.HostSequences([l.strip() for l in open(lst) if l.strip()])
    r = engine.build(hs.batch, k, B, n)
    want = (native.result_frag_bytes(r), native.result_class_words(r), native.result_class_offsets(r))
    shards = [sharded.build_shard(engine, hs.batch, k, B, n, rank, world) for rank in range(world)]
    assert sum(len(s[0]) for s in shards) == len(want[0])
    frag, w, o, bits = sharded.merge_shards(shards)
    assert frag == want[0]
    assert np.array_equal(w, want[1]) and bits == r.class_bits
    assert np.array_equal(o, want[2])


@pytest.mark.parametrize("k,world", [(31, 2), (31, 3), (63, 2)])
def test_split_by_file_merges_to_single(engine, tmp_path, k, world):
    """Phase 1 split by input file: each rank's drop-in phase 1 reads only its
    files (first_color = its first file), the records of each bucket range are
    merged from all ranks (cdbg_merge_bucket_records; the all-to-all that
    carries them is covered on CPU by test_sharded_files.py), each range runs
    the drop-in phase 2, and the merged shards equal the single drop-in build
    byte for byte -- its bucket records too."""
    import os
    p = synth.make_params(seed=60 + k + world, len_min=30000, len_max=90000, div_min=0.001, div_max=0.02,
                          indels=8, mobile_pool=3, mobile_min=800, mobile_max=2000, contigs_min=1,
                          contigs_max=12, contigs_log=1, lowercase_runs=1, n_runs=1,
                          tandem_frac=0.01 if k > 31 else 0.0)
    n, B = 10, 256
    files = [l.strip() for l in open(synth.write_fasta(p, n, str(tmp_path / "in"), gzip_level=1)) if l.strip()]
    single = str(tmp_path / "single")
    engine.phase1(files, k, B, single)
    engine.phase2(single, B, k, n, os.path.join(single, "frag_unitigs.bin"), os.path.join(single, "out.color_sets"))
    want = sharded.shard_from_phase2(os.path.join(single, "frag_unitigs.bin"), os.path.join(single, "out.color_sets"))
    raw_all, off_all = sharded.read_bucket_dir(single, B)
    runs = []
    for rank in range(world):
        f0, f1 = sharded.file_range(n, rank, world)
        d = str(tmp_path / ("p1_%d" % rank))
        engine.phase1(files[f0:f1], k, B, d, first_color=f0)
        runs.append(sharded.read_bucket_dir(d, B))
    shards = []
    for rank in range(world):
        lo, hi = sharded.shard_range(B, rank, world)
        sources = [(raw[int(off[lo]):int(off[hi])], (off[lo:hi + 1] - off[lo]).astype(np.uint64)) for raw, off in runs]
        data, moff = sharded.merge_bucket_records(sources, B, lo, hi)
        assert data == raw_all[int(off_all[lo]):int(off_all[hi])]
        md = str(tmp_path / ("merged_%d" % rank))
        sharded.write_bucket_dir(md, lo, data, moff)
        engine.phase2(md, B, k, n, os.path.join(md, "frag_unitigs.bin"), os.path.join(md, "out.color_sets"))
        shards.append(sharded.shard_from_phase2(os.path.join(md, "frag_unitigs.bin"),
                                                os.path.join(md, "out.color_sets")))
    frag, w, o, bits = sharded.merge_shards(shards)
    assert frag == want[0]
    assert np.array_equal(w, want[1]) and bits == want[2]
    assert np.array_equal(o, want[3])
