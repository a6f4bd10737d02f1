"""CPU: the library's host reader (cdbg_read_sequences: gzip inflate, then
FASTA through a memchr line scan, or FASTQ through the general record
parser) gives the records kseq_read gives (external/kseq.h, as the
reference's seq_reader::next uses it, phase1_bucket_write/seq_reader.hpp:66):
the rules restated below in Python, on inputs that probe every edge."""
import gzip
import os

import numpy as np
import pytest

from cdbg_gpu import native


def _kseq(data):
    """Records of a FASTA/FASTQ byte string by kseq_read's rules."""
    out, p, n, last = [], 0, len(data), 0
    while True:
        if last == 0:
            while p < n and data[p] not in b">@":
                p += 1
            if p >= n:
                return out
            last = data[p]
            p += 1
        if p >= n:
            return out
        c = 0
        while p < n and data[p] not in b" \t\n\v\f\r":
            p += 1
        if p < n:
            c = data[p]
            p += 1
        if c != ord("\n"):
            while p < n:
                p += 1
                if data[p - 1] == ord("\n"):
                    break
        seq, cc = bytearray(), -1
        while p < n:
            cc = data[p]
            p += 1
            if cc in b">+@":
                break
            cc = -1
            if data[p - 1] == ord("\n"):
                continue
            e = p - 1
            while p < n and data[p] != ord("\n"):
                p += 1
            seq += data[e:p]
            if p < n:
                p += 1
        if cc in (ord(">"), ord("@")):
            last = cc
        if cc != ord("+"):
            out.append(bytes(seq))
            if cc == -1:
                return out
            continue
        while p < n and data[p] != ord("\n"):
            p += 1
        if p >= n:
            return out
        p += 1
        q = 0
        while p < n:
            qc = data[p]
            p += 1
            if q >= len(seq):
                break
            if 33 <= qc <= 127:
                q += 1
        last = 0
        if q != len(seq):
            return out
        out.append(bytes(seq))


CASES = [
    b">a\nACGT\nacgt\n>b desc\n\nNNAC\n",
    b"junk\n>a x y\nAC\r\nGT\n>b\n",
    b">only",
    b">",
    b">a\nAC\n@b\nGG\n+\nII\n>c\nTT\n",
    b"@r1\nACGT\n+\nIIII\n@r2\nAC\n+r2\nII\n",
    b">a\nACG\n+x\nTT\n",
    b"\n\n>a\n\n\nACGT\n\n>b\nC",
]


@pytest.mark.parametrize("i", range(len(CASES)))
@pytest.mark.parametrize("gz", [False, True])
def test_reader_follows_kseq(tmp_path, i, gz):
    data = CASES[i]
    p = str(tmp_path / ("f.fa" + (".gz" if gz else "")))
    with open(p, "wb") as f:
        f.write(gzip.compress(data) if gz else data)
    hs = native.HostSequences([p])
    seq, off = hs.seq_bytes(), hs.offsets()
    got = [seq[int(off[j]):int(off[j + 1])] for j in range(len(off) - 1)]
    assert got == _kseq(data)


def test_reader_random_fasta(tmp_path):
    rng = np.random.default_rng(3)
    recs = []
    for j in range(200):
        L = int(rng.integers(0, 500))
        s = bytes(rng.choice(list(b"ACGTNacgt"), size=L).tolist())
        width = int(rng.integers(1, 120))
        body = b"\n".join(s[x:x + width] for x in range(0, len(s), width))
        recs.append(b">r%d c\n" % j + body + (b"\n" if rng.random() < 0.8 else b"\n\n"))
    data = b"".join(recs)
    p = str(tmp_path / "r.fa.gz")
    with open(p, "wb") as f:
        f.write(gzip.compress(data))
    hs = native.HostSequences([p, p])
    seq, off = hs.seq_bytes(), hs.offsets()
    got = [seq[int(off[j]):int(off[j + 1])] for j in range(len(off) - 1)]
    assert got == _kseq(data) * 2
    assert list(hs.colors()) == [0] * (len(got) // 2) + [1] * (len(got) // 2)
