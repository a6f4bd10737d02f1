"""GPU: the device reader (cdbg_tuning.gpu_inflate).

* The device gzip decoder (cdbg_gpu_gunzip, the decoder the device reader
  runs) against zlib on streams of every DEFLATE block type and zlib
  strategy, codes longer than the one-lookup table, long and overlapping
  matches, multi-member files and gzip headers with every optional field;
  truncated, corrupt and oversized streams are refused (status 2 or 1), never
  decoded differently.
* Builds whose files are read by the device (gpu_inflate = 1) against the
  same builds read by the host reader (gpu_inflate = 2), on collections and
  on FASTA files written to hit the record rules' edge cases; FASTQ and
  multi-member inputs go back to the host reader with the same outputs.
"""
import filecmp
import gzip
import os
import struct
import zlib

import numpy as np
import pytest

from cdbg_gpu import synth

pytestmark = pytest.mark.gpu


def _gz(data, level=6, strategy=zlib.Z_DEFAULT_STRATEGY, mem=8):
    c = zlib.compressobj(level, zlib.DEFLATED, 31, mem, strategy)
    return c.compress(data) + c.flush()


def _member(data, flags=0, extra=b"", name=b"", comment=b"", level=6):
    """A gzip member with the optional header fields set by hand (RFC 1952)."""
    c = zlib.compressobj(level, zlib.DEFLATED, -15)
    body = c.compress(data) + c.flush()
    h = bytearray(b"\x1f\x8b\x08" + bytes([flags]) + b"\x00\x00\x00\x00\x00\xff")
    if flags & 4:
        h += struct.pack("<H", len(extra)) + extra
    if flags & 8:
        h += name + b"\x00"
    if flags & 16:
        h += comment + b"\x00"
    if flags & 2:
        h += struct.pack("<H", zlib.crc32(bytes(h)) & 0xffff)
    return bytes(h) + body + struct.pack("<II", zlib.crc32(data) & 0xffffffff, len(data) & 0xffffffff)


def _dna(rng, n, lower=0.0):
    s = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=n)
    if lower:
        m = rng.random(n) < lower
        s[m] |= 0x20
    return s.tobytes()


def _cases():
    rng = np.random.default_rng(5)
    dna = _dna(rng, 600_000)
    rep = (_dna(rng, 3000) * 200)[:500_000]            # long matches at distance 3000
    homo = b"A" * 100_000 + b"AC" * 50_000 + dna[:10_000]  # distance 1 and 2 (overlapping copies)
    # a skewed byte distribution: Huffman codes up to 15 bits
    p = 0.5 ** (np.arange(256) / 12.0)
    skew = rng.choice(256, size=400_000, p=p / p.sum()).astype(np.uint8).tobytes()
    noise = rng.integers(0, 256, size=300_000, dtype=np.uint8).tobytes()  # stored blocks
    far = dna[:40_000] + _dna(rng, 20_000) + dna[:40_000]                # distances near 32 KiB
    fasta = b"".join(b">g%d some header\n" % i + b"\n".join(dna[j:j + 60] for j in range(i * 6000, i * 6000 + 6000, 60))
                     + b"\n" for i in range(50))
    out = []
    for data in (b"", b"A", dna, rep, homo, skew, noise, far, fasta):
        out.append(_gz(data, 1))
        out.append(_gz(data, 6))
    for strat in (zlib.Z_FILTERED, zlib.Z_HUFFMAN_ONLY, zlib.Z_RLE, zlib.Z_FIXED):
        out.append(_gz(dna[:200_000] + skew[:50_000], 6, strat))
    out.append(_gz(dna, 0))                               # stored only
    out.append(_gz(dna[:300_000], 9, mem=9))
    out.append(_gz(fasta[:1000], 1) + _gz(fasta[1000:5000], 9))  # two members
    out.append(_member(dna[:70_000], flags=4 | 8 | 16 | 2, extra=b"AB\x04\x00wxyz", name=b"g.fa",
                       comment=b"a comment"))
    out.append(_member(b"", flags=8, name=b"empty"))
    return out


def test_gunzip_matches_zlib(engine):
    streams = _cases()
    want = [gzip.decompress(s) if s else b"" for s in streams]
    got = engine.gunzip(streams, [len(w) + 64 for w in want])
    for i, ((st, data), w) in enumerate(zip(got, want)):
        if not streams[i]:
            assert st == 2  # no gzip header at all
            continue
        assert st == 0, i
        assert data == w, i


def test_gunzip_refuses_bad_streams(engine):
    rng = np.random.default_rng(9)
    dna = _dna(rng, 100_000)
    good = _gz(dna, 6)
    trunc = good[: len(good) // 2]
    badmagic = b"\x1f\x8c" + good[2:]
    bad_isize = good[:-4] + struct.pack("<I", len(dna) + 1)
    flipped = bytearray(good)
    flipped[10] ^= 0xff  # the first block header: invalid codes or a wrong size
    trailing = good + b"\x00\x01\x02"
    res = engine.gunzip([trunc, badmagic, bad_isize, bytes(flipped), trailing, good],
                        [len(dna) + 64] * 5 + [len(dna) - 1])
    for i, (st, _) in enumerate(res[:5]):
        # refused: not a stream it accepts, or (a corrupted one) decoding
        # past its region before the error shows
        assert st == 2 or (i == 3 and st == 1), (i, st)
    assert res[5][0] == 1  # more bytes than the region holds


# ---------------------------------------------------------------- builds
def _build(engine, files, k, B, d, mode):
    engine.set_tuning(gpu_inflate=mode)
    frag, cs = os.path.join(d, "frag%d.bin" % mode), os.path.join(d, "cs%d" % mode)
    r = engine.build_files(files, k, B, frag, cs, host_threads=4)
    engine.set_tuning()
    return frag, cs, r


def _same_builds(engine, files, k, B, tmp_path):
    d = str(tmp_path)
    f1, c1, r1 = _build(engine, files, k, B, d, 1)
    f2, c2, r2 = _build(engine, files, k, B, d, 2)
    assert filecmp.cmp(f1, f2, shallow=False)
    assert filecmp.cmp(c1, c2, shallow=False)
    assert r1.n_kmers == r2.n_kmers and r1.n_kmers > 0
    assert r1.total_seq_bytes == r2.total_seq_bytes
    return r1


@pytest.mark.parametrize("k,level", [(31, 1), (63, 6)])
def test_device_reader_equals_host_reader(engine, tmp_path, k, level):
    p = synth.make_params(seed=70 + k, len_min=40000, len_max=150000, div_min=0.001, div_max=0.02, indels=10,
                          mobile_pool=3, mobile_min=1000, mobile_max=3000, contigs_min=1, contigs_max=20,
                          contigs_log=1, lowercase_runs=1, n_runs=1, tandem_frac=0.01 if k > 31 else 0.0)
    lst = synth.write_fasta(p, 14, str(tmp_path / "in"), gzip_level=level)
    files = [l.strip() for l in open(lst) if l.strip()]
    _same_builds(engine, files, k, 256, tmp_path)


def _write(path, text, gz=True):
    with open(path, "wb") as f:
        f.write(_gz(text, 1) if gz else text)
    return path


def test_device_reader_record_rules(engine, tmp_path):
    rng = np.random.default_rng(12)
    seq = [_dna(rng, 5000, lower=0.05) for _ in range(12)]
    hdr_acgt = b"ACGT" * 20
    texts = [
        # junk and a '>' in the middle of the first line before the first header
        b"junk ACGTACGTACGTACGTACGTACGTACGTACGTACGT>first " + hdr_acgt + b"\n" + seq[0] + b"\n",
        # empty lines, CRLF line ends, no final newline
        b">a\r\n" + seq[1][:2000] + b"\r\n\r\n" + seq[1][2000:] + b"\r\n>b\n\n\n" + seq[2],
        # header text made of bases (must not become k-mers), N runs, a '>' inside a line
        b">" + hdr_acgt + b" " + hdr_acgt + b"\n" + seq[3][:1000] + b"NNNNN" + seq[3][1000:3000] + b">" +
        seq[3][3000:] + b"\n",
        # records with no sequence, and lines of many lengths
        b">e1\n>e2\n\n>x\n" + b"\n".join(seq[4][i:i + L] for i, L in zip(range(0, 5000, 500), [1, 7, 60, 500] * 3))
        + b"\n>e3\n",
        # no header at all: nothing
        seq[5] + b"\n",
        b"",
        # many short records
        b"".join(b">r%d\n" % i + seq[6][i * 100:(i + 1) * 100] + b"\n" for i in range(50)),
        # a long single line
        b">long\n" + b"".join(seq[7:12]) + b"\n",
    ]
    files = [_write(str(tmp_path / ("f%d.fa.gz" % i)), t) for i, t in enumerate(texts)]
    # one plain file among the gzip ones
    files.append(_write(str(tmp_path / "plain.fa"), b">p\n" + seq[8] + b"\n", gz=False))
    _same_builds(engine, files, 31, 64, tmp_path)


def test_fastq_and_multimember_go_back_to_the_host_reader(engine, tmp_path):
    rng = np.random.default_rng(13)
    s = [_dna(rng, 4000) for _ in range(4)]
    fa = [_write(str(tmp_path / ("a%d.fa.gz" % i)), b">s\n" + s[i] + b"\n") for i in range(3)]
    fq = _write(str(tmp_path / "q.fq.gz"), b"@r1\n" + s[3] + b"\n+\n" + b"I" * len(s[3]) + b"\n")
    _same_builds(engine, fa + [fq], 31, 64, tmp_path)
    # a file of two members: its size field covers the second one only
    mm = str(tmp_path / "mm.fa.gz")
    with open(mm, "wb") as f:
        f.write(_gz(b">m1\n" + s[0] + b"\n", 1) + _gz(b">m2\n" + s[1][:100] + b"\n", 1))
    _same_builds(engine, fa + [mm], 31, 64, tmp_path)


def test_device_reader_dropin_phase1(engine, oracle, tmp_path):
    p = synth.make_params(seed=91, len_min=30000, len_max=90000, div_min=0.001, div_max=0.02, indels=8,
                          mobile_pool=3, mobile_min=800, mobile_max=2000, contigs_min=1, contigs_max=12,
                          contigs_log=1, lowercase_runs=1, n_runs=1)
    lst = synth.write_fasta(p, 10, str(tmp_path / "in"), gzip_level=1)
    files = [l.strip() for l in open(lst) if l.strip()]
    from cdbg_gpu import formats
    B = 128
    engine.set_tuning(gpu_inflate=1)
    try:
        gb = tmp_path / "gb"
        os.makedirs(gb)
        st, _ = engine.phase1(files, 31, B, str(gb))
    finally:
        engine.set_tuning()
    ob = tmp_path / "ob"
    os.makedirs(ob)
    ns, nk = oracle.phase1(lst, 31, B, bucket_dir=str(ob))
    assert (st.n_supers, st.n_kmers) == (ns, nk)
    for b in range(B):
        g, o = str(gb / ("bucket_%d.bin" % b)), str(ob / ("bucket_%d.bin" % b))
        assert formats.read_bucket_raw(g) == formats.read_bucket_raw(o), b
