"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cdbg-builder_b200")
for p in (PKG, ROOT, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


def ref_bin(name, k):
    p = os.path.join(REF_DIR, name + ("-largek" if k > 31 else ""))
    return p if os.path.exists(p) else None


class Oracle:
    """ctypes view of oracle/liboracle.so (the CPU restatement; checker only)."""

    def __init__(self):
        L = ctypes.CDLL(ORACLE_LIB)
        u32, u64, cp, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_void_p
        L.oracle_phase1.argtypes = [cp, u32, u32, u32, cp, cp, vp, vp]
        L.oracle_phase2.argtypes = [cp, u32, u32, u32, cp, vp, vp, vp]
        L.oracle_last_error.restype = cp
        L.oracle_bucket_kmers.argtypes = [cp, u32, u32, u32, vp]
        L.oracle_best_m.argtypes = [u32]
        L.oracle_best_m.restype = u32
        L.oracle_mhashes.argtypes = [vp, u32, u32, vp]
        L.oracle_kminus1_minimizers.argtypes = [vp, u32, u32, u32, vp]
        L.oracle_super_hash.argtypes = [vp, u32]
        L.oracle_super_hash.restype = u64
        self.L = L

    def phase1(self, filelist, k, B, dump=None, bucket_dir=None, m=0):
        ns, nk = ctypes.c_uint64(), ctypes.c_uint64()
        rc = self.L.oracle_phase1(filelist.encode(), k, m, B, dump.encode() if dump else None,
                                  bucket_dir.encode() if bucket_dir else None, ctypes.byref(ns),
                                  ctypes.byref(nk))
        if rc:
            raise RuntimeError(self.L.oracle_last_error().decode())
        return ns.value, nk.value

    def bucket_kmers(self, filelist, k, B, m=0):
        """k-mer occurrences per bucket, before deduplication."""
        import numpy as np
        c = np.zeros(B, dtype=np.uint64)
        if self.L.oracle_bucket_kmers(filelist.encode(), k, m, B, c.ctypes.data) != 0:
            raise RuntimeError(self.L.oracle_last_error().decode())
        return c

    def phase2(self, bucket_dir, B, k, C, out_dir):
        os.makedirs(out_dir, exist_ok=True)
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        rc = self.L.oracle_phase2(bucket_dir.encode(), B, k, C, out_dir.encode(), ctypes.byref(a),
                                  ctypes.byref(b), ctypes.byref(c))
        if rc:
            raise RuntimeError(self.L.oracle_last_error().decode())
        return dict(fragments=a.value, num_color_sets=b.value, total_seq_bytes=c.value)


@pytest.fixture(scope="session")
def oracle():
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle/liboracle.so not built")
    return Oracle()


@pytest.fixture(scope="session")
def engine():
    from cdbg_gpu import Engine
    e = Engine(0)
    yield e
    e.close()


def golden_case(name):
    import json
    d = os.path.join(GOLDEN, name)
    meta = json.load(open(os.path.join(d, "meta.json")))
    return d, meta


def golden_filelist(case_dir, tmp_path):
    """Absolute filenames list for a golden case's inputs."""
    names = [l.strip() for l in open(os.path.join(case_dir, "in", "filenames.txt")) if l.strip()]
    p = os.path.join(str(tmp_path), "files.txt")
    with open(p, "w") as f:
        for n in names:
            f.write(os.path.join(case_dir, "in", n) + "\n")
    return p, [os.path.join(case_dir, "in", n) for n in names]


def run_ref(args):
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return r.stdout


def read_round_file(path):
    """Frames of a stitch round file ([u32 raw][u32 comp][bytes]... [u32 0]),
    decompressed with the system LZ4 library: a list of raw frame bytes."""
    import struct
    L = ctypes.CDLL("liblz4.so.1")
    L.LZ4_decompress_safe.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    data = open(path, "rb").read()
    frames, p = [], 0
    while True:
        (u,) = struct.unpack_from("<I", data, p)
        p += 4
        if u == 0:
            break
        (c,) = struct.unpack_from("<I", data, p)
        p += 4
        dst = ctypes.create_string_buffer(u)
        assert L.LZ4_decompress_safe(data[p:p + c], dst, c, u) == u, path
        frames.append(dst.raw)
        p += c
    assert p == len(data), "bytes after the end mark in " + path
    return frames


def round0_files(d, num_buckets):
    """{bucket: file bytes} of the stitch_r0_b<b>.bin files in d."""
    out = {}
    for b in range(num_buckets):
        p = os.path.join(d, "stitch_r0_b%d.bin" % b)
        if os.path.exists(p):
            out[b] = open(p, "rb").read()
    return out


_ACGT = bytes(b"ACGT"[i & 3] for i in range(256))


def synth_frags(seed, n, k, max_runs=4, max_m=20, p_foreign=0.2, p_closed=0.3):
    """n random frag records (unitig_spill.hpp:491-522 layout) with the shapes
    the seed branches on: closed and open (left, right, both) fragments, color
    runs of several k-mers, COLOR_RUN_FOREIGN runs at the ends and inside,
    closed fragments without runs.  Each sequence has sum(num_kmers) + k - 1
    ACGT bases, and an open one at least k."""
    import random
    import struct
    r = random.Random(seed)
    out = bytearray()
    for _ in range(n):
        closed = r.random() < p_closed
        of = 0 if closed else r.choice((1, 2, 3))
        nr = r.randint(0 if closed else 1, max_runs)
        runs = [((2 ** 64 - 1) if r.random() < p_foreign else r.randrange(1 << 20), r.randint(1, max_m))
                for _ in range(nr)]
        ln = sum(m for _, m in runs) + k - 1 if runs else k - 1
        seq = r.randbytes(ln).translate(_ACGT)
        out += struct.pack("<BI", of, nr)
        for cid, m in runs:
            out += struct.pack("<QI", cid, m)
        out += struct.pack("<I", ln) + seq
    return bytes(out)
