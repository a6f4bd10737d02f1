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
