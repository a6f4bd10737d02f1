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
