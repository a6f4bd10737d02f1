"""GPU: the allocation-free super-k-mer entry point (cdbg_gpu_supers_noalloc).

Some callers cannot allocate device memory (their host application owns all
of it, or allocation is not allowed where they run), so this entry point
takes every buffer from the caller and keeps its working memory in a fixed
device array.  This test calls it through the C-ABI on two calls in a row
and checks each result, super-k-mer by super-k-mer, against the existing
entry point cdbg_gpu_dump_supers on the same sequences.  It lives in a file
of its own that pytest collects last.
"""
import ctypes
import os
import struct

import numpy as np
import pytest

from cdbg_gpu import native, synth

pytestmark = pytest.mark.gpu


def _runs(seq, off, k):
    """ACGT runs >= k of every sequence: (codes uint8 array, color) list."""
    code = np.full(256, 255, dtype=np.uint8)
    for ch, v in zip(b"ACGTacgt", [0, 1, 2, 3, 0, 1, 2, 3]):
        code[ch] = v
    c = code[np.frombuffer(seq, dtype=np.uint8)]
    runs = []
    for i in range(len(off) - 1):
        s = c[int(off[i]):int(off[i + 1])]
        valid = s != 255
        edges = np.flatnonzero(np.diff(np.concatenate(([0], valid.astype(np.int8), [0]))))
        for a, b in zip(edges[0::2], edges[1::2]):
            if b - a >= k:
                runs.append((s[a:b], i))
    return runs


def _pack(runs):
    soff, lens, total = [], [], 0
    for r, _ in runs:
        soff.append(total)
        lens.append(len(r))
        total += (len(r) + 31) // 32 * 32
    words = np.zeros(total // 32 + 8, dtype=np.uint64)
    for (r, _), so in zip(runs, soff):
        v = np.zeros((len(r) + 31) // 32 * 32, dtype=np.uint64)
        v[:len(r)] = r
        shifts = (2 * (np.arange(len(v)) % 32)).astype(np.uint64)
        w = np.bitwise_or.reduce((v << shifts).reshape(-1, 32), axis=1)
        words[so // 32: so // 32 + len(w)] = w
    return words, np.array(soff, dtype=np.uint64), np.array(lens, dtype=np.uint32)


def _dump_bytes(words, start, ln, color, flags, bucket):
    """The layout cdbg_gpu_dump_supers writes, rebuilt from the outputs."""
    out = [struct.pack("<Q", len(start))]
    for s, l, c, f, b in zip(start, ln, color, flags, bucket):
        pk = bytearray((int(l) + 3) // 4)
        for i in range(int(l)):
            p = int(s) + i
            base = (int(words[p >> 5]) >> (2 * (p & 31))) & 3
            pk[i >> 2] |= base << (2 * (i & 3))
        out.append(struct.pack("<IBII", int(b), int(f), int(c), int(l)) + bytes(pk))
    return b"".join(out)


def _case(tmp_path, seed, k):
    p = synth.make_params(seed=seed, len_min=6000, len_max=15000, div_min=0.002, div_max=0.02,
                          indels=3, mobile_pool=2, mobile_min=300, mobile_max=900, contigs_min=1,
                          contigs_max=6, contigs_log=1, lowercase_runs=1, n_runs=1)
    lst = synth.write_fasta(p, 4, str(tmp_path / ("in%d" % seed)))
    files = [l.strip() for l in open(lst) if l.strip()]
    hs = native.HostSequences(files)
    seq, off, colors = hs.seq_bytes(), hs.offsets(), hs.colors()
    runs = _runs(seq, off, k)
    words, soff, lens = _pack(runs)
    rcol = np.array([colors[i] for _, i in runs], dtype=np.uint32)
    return hs, words, soff, lens, rcol


def test_noalloc_matches_dump_supers_twice(engine, tmp_path):
    import torch
    L = native.lib()
    k, m, B = 31, native.best_m(31), 256
    for call, seed in enumerate((3, 4)):  # two calls in a row, different inputs
        hs, words, soff, lens, rcol = _case(tmp_path, seed, k)
        ref = str(tmp_path / ("ref%d.bin" % call))
        n_ref = engine.dump_supers(hs.batch, k, m, B, ref)
        dw = torch.from_numpy(words.view(np.int64)).cuda()
        ds = torch.from_numpy(soff.view(np.int64)).cuda()
        dl = torch.from_numpy(lens.view(np.int32)).cuda()
        dc = torch.from_numpy(rcol.view(np.int32)).cuda()
        cap = n_ref + 16
        o_start = torch.zeros(cap, dtype=torch.int64, device="cuda")
        o_len, o_col, o_fl, o_bk = (torch.zeros(cap, dtype=torch.int32, device="cuda") for _ in range(4))
        n = ctypes.c_uint64()
        torch.cuda.synchronize()
        rc = L.cdbg_gpu_supers_noalloc(dw.data_ptr(), ds.data_ptr(), dl.data_ptr(), dc.data_ptr(),
                                       len(lens), k, m, B, o_start.data_ptr(), o_len.data_ptr(),
                                       o_col.data_ptr(), o_fl.data_ptr(), o_bk.data_ptr(), cap,
                                       ctypes.byref(n), None)
        assert rc == 0, L.cdbg_last_error()
        assert n.value == n_ref
        got = _dump_bytes(words, o_start.cpu().numpy()[:n.value], o_len.cpu().numpy()[:n.value],
                          o_col.cpu().numpy()[:n.value], o_fl.cpu().numpy()[:n.value],
                          o_bk.cpu().numpy()[:n.value])
        assert got == open(ref, "rb").read(), "call %d differs" % call


def _call(L, words_ptr, soff, lens, k, m=12, B=64, cap=16):
    import torch
    ds = torch.from_numpy(np.asarray(soff, dtype=np.uint64).view(np.int64)).cuda()
    dl = torch.from_numpy(np.asarray(lens, dtype=np.uint32).view(np.int32)).cuda()
    dc = torch.zeros(len(lens), dtype=torch.int32, device="cuda")
    out = torch.zeros(cap, dtype=torch.int64, device="cuda")
    n = ctypes.c_uint64()
    rc = L.cdbg_gpu_supers_noalloc(words_ptr, ds.data_ptr(), dl.data_ptr(), dc.data_ptr(), len(lens), k, m, B,
                                   out.data_ptr(), out.data_ptr(), out.data_ptr(), out.data_ptr(),
                                   out.data_ptr(), cap, ctypes.byref(n), None)
    torch.cuda.synchronize()
    return rc


def test_noalloc_rejects_bad_inputs_then_recovers(engine, tmp_path):
    """Inputs past the fixed working array, runs shorter than k and a
    misaligned stream are refused with an error before any tile kernel reads
    them; a valid call afterwards still matches the allocating entry point."""
    import torch
    L = native.lib()
    k = 31
    # one run of 1.1M bases: few runs, but more than 512 tiles of 2048 (k-1)-mers
    words = torch.zeros(1_100_000 // 32 + 16, dtype=torch.int64, device="cuda")
    assert _call(L, words.data_ptr(), [0], [1_100_000], k) != 0
    assert b"tiles" in L.cdbg_last_error()
    # a run of k - 1 bases has no k-mer
    assert _call(L, words.data_ptr(), [0, 64], [40, k - 1], k) != 0
    assert b"shorter than k" in L.cdbg_last_error()
    # the stream must be 16-byte aligned (8 bytes into a buffer is not)
    assert _call(L, words.data_ptr() + 8, [0], [40], k) != 0
    assert b"aligned" in L.cdbg_last_error()
    test_noalloc_matches_dump_supers_twice(engine, tmp_path)


def test_noalloc_rejects_oversized_input(engine):
    import torch
    L = native.lib()
    k = 31
    # 600 runs of 40 bases: more runs than the 512-tile working array allows
    lens = np.full(600, 40, dtype=np.uint32)
    soff = (np.arange(600, dtype=np.uint64) * 64)
    words = torch.zeros(600 * 2 + 8, dtype=torch.int64, device="cuda")
    ds = torch.from_numpy(soff.view(np.int64)).cuda()
    dl = torch.from_numpy(lens.view(np.int32)).cuda()
    dc = torch.zeros(600, dtype=torch.int32, device="cuda")
    out = torch.zeros(16, dtype=torch.int64, device="cuda")
    n = ctypes.c_uint64()
    rc = L.cdbg_gpu_supers_noalloc(words.data_ptr(), ds.data_ptr(), dl.data_ptr(), dc.data_ptr(), 600, k,
                                   12, 64, out.data_ptr(), out.data_ptr(), out.data_ptr(), out.data_ptr(),
                                   out.data_ptr(), 16, ctypes.byref(n), None)
    assert rc != 0 and b"512" in L.cdbg_last_error()
