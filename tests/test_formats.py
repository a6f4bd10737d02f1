"""CPU: artifact readers and the invariants of the golden outputs."""
import os

import pytest

from conftest import golden_case
from cdbg_gpu import formats

CASES = ["tiny_k31", "tiny_k63", "tiny_skew_fq"]


@pytest.mark.parametrize("case", CASES)
def test_frag_invariants(case):
    d, meta = golden_case(case)
    k = meta["k"]
    frags = formats.read_frags(os.path.join(d, "frag_unitigs.bin"))
    assert len(frags) == int(meta["phase2"]["fragments"])
    assert sum(len(s) for _, _, s in frags) == int(meta["phase2"]["total_seq_bytes"])
    for fl, runs, seq in frags:
        assert fl <= 3
        assert sum(n for _, n in runs) == len(seq) - k + 1  # bucket_walker.hpp:89-95
        assert set(seq) <= set("ACGT")


@pytest.mark.parametrize("case", CASES)
def test_color_sets_decode(case):
    d, meta = golden_case(case)
    C, words, offsets, classes = formats.read_color_sets(os.path.join(d, "out.color_sets"))
    assert C == meta["num_colors"]
    assert len(classes) == int(meta["metadata"]["num_color_sets"])
    seen = set()
    for c in classes:
        assert c == sorted(set(c)) and c and all(0 <= x < C for x in c)
        seen.add(tuple(c))
    assert len(seen) == len(classes)  # classes are distinct
    frags = formats.read_frags(os.path.join(d, "frag_unitigs.bin"))
    used = {cid for _, runs, _ in frags for cid, _ in runs if cid != formats.FOREIGN}
    assert used == set(range(len(classes)))


def test_delta_roundtrip():
    import numpy as np
    vals = [0, 1, 2, 3, 7, 8, 100, 1023, 1024, 65535, 2**31, 2**32 - 1]
    # encode with a tiny Python writer following the same definition
    bits = []

    def put(x, n):
        for i in range(n):
            bits.append((x >> i) & 1)

    for x in vals:
        y = x + 1
        l = y.bit_length() - 1
        L1 = l + 1
        ll = L1.bit_length() - 1
        put(0, ll)
        put(1, 1)
        put(L1, ll)
        put(y, l)
    words = np.zeros((len(bits) + 63) // 64 + 1, dtype=np.uint64)
    for i, b in enumerate(bits):
        if b:
            words[i >> 6] |= np.uint64(1) << np.uint64(i & 63)
    r = formats._Bits(words, 0)
    assert [formats.read_delta(r) for _ in vals] == vals
