"""GPU: the performance knobs (bucket-batch split threshold, minimizer tile,
heavy-record bitmap threshold, k-mer table slots per occurrence) and the
autotuner never change outputs."""
import numpy as np
import pytest

from cdbg_gpu import native, synth

pytestmark = pytest.mark.gpu


def _batch(seed, n, **kw):
    base = dict(len_min=40000, len_max=160000, div_min=0.001, div_max=0.02, indels=5, mobile_pool=3,
                mobile_min=500, mobile_max=2000, contigs_min=1, contigs_max=10, contigs_log=1, lowcomp_frac=0.1,
                lowercase_runs=1, n_runs=1)
    base.update(kw)
    seq, lens, per = synth.collection(synth.make_params(seed=seed, **base), n)
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    return native.array_batch(seq, off, np.repeat(np.arange(n, dtype=np.uint32), per))


def _out(engine, b, k, B, n):
    r = engine.build(b, k, B, n)
    return native.result_frag_bytes(r), native.result_class_words(r), native.result_class_offsets(r)


@pytest.mark.parametrize("k", [31, 63])
def test_knobs_do_not_change_outputs(k):
    n, B = 40, 512
    b = _batch(71 + k, n)
    e = native.Engine(0)
    try:
        want = _out(e, b, k, B, n)
        for t in (dict(minimizer_tile=1024), dict(minimizer_tile=2048), dict(heavy_colors=1),
                  dict(heavy_colors=100000),
                  dict(batch_occ=1 << 12), dict(batch_occ=1, minimizer_tile=1024, heavy_colors=16),
                  dict(table_slots_q=5), dict(table_slots_q=16), dict(table_slots_q=5, batch_occ=1 << 14),
                  dict(union_lists=1, heavy_colors=1), dict(table_group_mb=1), dict(table_group_mb=1024),
                  dict(radix_bits=11), dict(radix_bits=11, table_group_mb=2, minimizer_tile=1024)):
            e.set_tuning(**t)
            got = _out(e, b, k, B, n)
            assert got[0] == want[0], t
            assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2]), t
    finally:
        e.close()


def test_autotune_keeps_outputs(engine):
    n, B = 30, 1024
    b = _batch(91, n)
    want = _out(engine, b, 31, B, n)
    e = native.Engine(0)
    try:
        t, ms = e.autotune(b, 31, B, n)
        assert ms > 0
        assert t["minimizer_tile"] in (1024, 2048, 4096)
        assert 5 <= t["table_slots_q"] <= 16
        assert e.tuning() == t
        got = _out(e, b, 31, B, n)
        assert got[0] == want[0]
        assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    finally:
        e.close()
