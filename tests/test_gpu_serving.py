"""GPU: the build server.  Requests submitted together (so they overlap on
the device under the HBM budget) return exactly what each build returns when
run alone; a memory-capped engine returns the same outputs as an uncapped one
(phase 2 just runs more, smaller bucket batches)."""
import numpy as np
import pytest

from cdbg_gpu import native, synth

pytestmark = pytest.mark.gpu


def _request(seed, n, k):
    extra = dict(tandem_frac=0.02, repeat_pool=3, repeat_min=300, repeat_max=800) if k > 31 else {}
    p = synth.make_params(seed=seed, len_min=30000, len_max=120000, div_min=0.001, div_max=0.02, indels=5,
                          mobile_pool=3, mobile_min=500, mobile_max=2000, contigs_min=1, contigs_max=8,
                          contigs_log=1, lowercase_runs=1, n_runs=1, **extra)
    seq, lens, per = synth.collection(p, n)
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    colors = np.repeat(np.arange(n, dtype=np.uint32), per)
    return native.array_batch(seq, off, colors), n, k


def _alone(engine, batch, n, k, B):
    r = engine.build(batch, k, B, n)
    return native.result_frag_bytes(r), native.result_class_words(r), native.result_class_offsets(r)


REQS = [(11, 3, 31), (12, 7, 63), (13, 2, 31), (14, 12, 31), (15, 5, 63), (16, 9, 31)]


def test_requests_in_the_mix_equal_requests_alone(engine):
    B = 256
    reqs = [_request(*r) for r in REQS]
    want = [_alone(engine, b, n, k, B) for b, n, k in reqs]
    with native.Server(0, slots=3, hbm_budget=24 << 30) as srv:
        ids = [srv.submit(b, k, B, n) for b, n, k in reqs]
        got = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2  # requests did overlap
    for g, (frag, words, offs) in zip(got, want):
        assert g["status"] == 0, g["error"]
        assert g["frag"] == frag
        assert np.array_equal(g["words"], words)
        assert np.array_equal(g["offsets"], offs)
        assert g["t_submit"] <= g["t_start"] <= g["t_done"]


def test_request_above_budget_runs_alone(engine):
    B = 128
    b, n, k = _request(21, 4, 31)
    want = _alone(engine, b, n, k, B)
    # the estimate (2 GiB floor) exceeds a 1.5 GiB budget: admitted alone, with the whole budget
    with native.Server(0, slots=2, hbm_budget=3 << 29) as srv:
        i1 = srv.submit(b, k, B, n)
        i2 = srv.submit(b, k, B, n)
        g1, g2 = srv.wait(i1), srv.wait(i2)
        st = srv.stats()
    assert st["peak_running"] == 1
    for g in (g1, g2):
        assert g["status"] == 0, g["error"]
        assert g["grant_bytes"] == 3 << 29
        assert g["frag"] == want[0]
        assert np.array_equal(g["words"], want[1])
    assert g2["t_start"] >= g1["t_done"]


def test_memory_capped_engine_matches_uncapped(engine):
    B = 256
    b, n, k = _request(31, 10, 31)
    want = _alone(engine, b, n, k, B)
    capped = native.Engine(0)
    try:
        capped.set_memory_limit(3 << 29)
        got = _alone(capped, b, n, k, B)
        _, peak = capped.memory()
    finally:
        capped.close()
    assert got[0] == want[0]
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    assert peak <= 3 << 29
