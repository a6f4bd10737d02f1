"""GPU: the stable 64-bit pair sort behind phase 1's (bucket, hash) record
order and phase 2's grouping of candidate color sets.  It runs four radix
passes over the top 32 key bits and then re-sorts only the runs whose keys
tie there but differ below; its order must equal a stable sort on the whole
key (numpy's stable argsort here), including the adversarial shapes where
many keys tie on the top bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(engine, keys):
    import torch
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    vals = np.arange(len(keys), dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    engine.sort_pairs_u64(dk.data_ptr(), dv.data_ptr(), len(keys))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 100_000, 3_000_000])
def test_random_keys(engine, n):
    rng = np.random.default_rng(n)
    _check(engine, rng.integers(0, 2**64, size=n, dtype=np.uint64))


def test_top_bits_tie_often(engine):
    """Few distinct top halves, many distinct bottom halves, duplicates."""
    rng = np.random.default_rng(5)
    n = 2_000_000
    hi = rng.integers(0, 64, size=n, dtype=np.uint64) << np.uint64(32)
    lo = rng.integers(0, 1000, size=n, dtype=np.uint64)
    _check(engine, hi | lo)


def test_one_huge_mixed_run(engine):
    """One top half everywhere (a run of the whole array) with two
    interleaved bottom values, plus a tail of unrelated keys."""
    rng = np.random.default_rng(9)
    n = 1_500_000
    k = np.full(n, 0xABCDEF01 << 32, dtype=np.uint64) | rng.integers(0, 2, size=n, dtype=np.uint64)
    k[-1000:] = rng.integers(0, 2**64, size=1000, dtype=np.uint64)
    _check(engine, k)


def test_constant_and_sorted_inputs(engine):
    _check(engine, np.full(50_000, 7, dtype=np.uint64))
    _check(engine, np.arange(200_000, dtype=np.uint64)[::-1] * np.uint64(0x9E3779B97F4A7C15))
    _check(engine, np.arange(200_000, dtype=np.uint64))


def test_sparse_ties_take_the_run_fixup(engine):
    """Top halves from 2^24 values over 2M keys: a few percent of the top
    runs are mixed (the re-sort path), most are single keys or exact
    duplicates (copies of one key keep their input order)."""
    rng = np.random.default_rng(11)
    n = 2_000_000
    hi = rng.integers(0, 1 << 24, size=n, dtype=np.uint64) << np.uint64(32)
    lo = rng.integers(0, 4, size=n, dtype=np.uint64) * np.uint64(0x10001)
    k = hi | lo
    k[1::5] = k[0::5]  # exact duplicates
    _check(engine, k)


@pytest.mark.parametrize("n", [5000, 1_000_000])
def test_eleven_bit_digits_give_the_same_order(engine, n):
    """The radix_bits knob (11-bit digits: 3 passes where 8-bit digits take
    4) sorts exactly alike."""
    rng = np.random.default_rng(n + 1)
    k = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    k[::3] = k[1::3][: len(k[::3])] if len(k[1::3]) >= len(k[::3]) else k[::3]
    engine.set_tuning(radix_bits=11)
    try:
        _check(engine, k)
        hi = rng.integers(0, 1 << 20, size=n, dtype=np.uint64) << np.uint64(32)
        _check(engine, hi | rng.integers(0, 8, size=n, dtype=np.uint64))
    finally:
        engine.set_tuning()
