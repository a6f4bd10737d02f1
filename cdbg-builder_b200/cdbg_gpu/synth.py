"""Synthetic pangenome workloads (ctypes binding to libcdbg_synth.so).

The presets restate the genome shapes of the five benchmark workloads:

* ``small``     10 genomes of ~5.0 Mbp, 0.5% SNPs, 20 indels, one 10-50 kbp
                mobile insert from a pool of 5, 1-3 contigs; k=31, -b 10.
* ``pangenome`` 1000 genomes of ~4.8 Mbp, 0.1-2% SNPs, 1-200 contigs
                (log-uniform), gzipped FASTA; k=31, -b 12.
* ``largek``    500 genomes as above plus 2% tandem repeats and 200 shared
                1-5 kbp repeats per genome; k=63, -b 12.
* ``skewed``    2000 genomes of 1-6 Mbp (log-uniform) with 10% homopolymer /
                dinucleotide content; k=31, -b 14.
* ``serving``   per-request collections: 2-300 genomes of 0.5-8 Mbp.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_HERE), "libcdbg_synth.so")


class SynthParams(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("len_min", ctypes.c_double), ("len_max", ctypes.c_double),
        ("div_min", ctypes.c_double), ("div_max", ctypes.c_double),
        ("indels", ctypes.c_uint32),
        ("mobile_pool", ctypes.c_uint32),
        ("mobile_min", ctypes.c_uint32), ("mobile_max", ctypes.c_uint32),
        ("repeat_pool", ctypes.c_uint32),
        ("repeats_per_genome", ctypes.c_uint32),
        ("contigs_min", ctypes.c_uint32), ("contigs_max", ctypes.c_uint32),
        ("contigs_log", ctypes.c_uint32),
        ("tandem_frac", ctypes.c_double),
        ("lowcomp_frac", ctypes.c_double),
        ("lowercase_runs", ctypes.c_uint32),
        ("n_runs", ctypes.c_uint32),
    ]


# name -> (params, num_genomes, k, buckets_log2)
PRESETS = {
    "small": (dict(len_min=5.0e6, len_max=5.0e6, div_min=0.005, div_max=0.005, indels=20,
                   mobile_pool=5, mobile_min=10000, mobile_max=50000,
                   contigs_min=1, contigs_max=3), 10, 31, 10),
    "pangenome": (dict(len_min=4.8e6, len_max=4.8e6, div_min=0.001, div_max=0.02, indels=20,
                       mobile_pool=5, mobile_min=10000, mobile_max=50000,
                       contigs_min=1, contigs_max=200, contigs_log=1), 1000, 31, 12),
    "largek": (dict(len_min=4.8e6, len_max=4.8e6, div_min=0.001, div_max=0.02, indels=20,
                    mobile_pool=5, mobile_min=10000, mobile_max=50000,
                    repeat_pool=50, repeats_per_genome=200, tandem_frac=0.02,
                    contigs_min=1, contigs_max=200, contigs_log=1), 500, 63, 12),
    "skewed": (dict(len_min=1.0e6, len_max=6.0e6, div_min=0.001, div_max=0.02, indels=20,
                    mobile_pool=5, mobile_min=10000, mobile_max=50000, lowcomp_frac=0.10,
                    contigs_min=1, contigs_max=200, contigs_log=1), 2000, 31, 14),
    "serving": (dict(len_min=0.5e6, len_max=8.0e6, div_min=0.001, div_max=0.02, indels=20,
                     mobile_pool=5, mobile_min=10000, mobile_max=50000,
                     contigs_min=1, contigs_max=200, contigs_log=1), 300, 31, 12),
}


def make_params(seed=1, **kw):
    p = SynthParams()
    p.seed = seed
    for name, _ in SynthParams._fields_:
        if name != "seed":
            setattr(p, name, type(getattr(p, name))(0))
    p.contigs_min = p.contigs_max = 1
    for key, v in kw.items():
        setattr(p, key, v)
    return p


def preset(name, seed=1, scale=1.0, **override):
    """Params of a preset; `scale` shrinks genome lengths (tests use < 1)."""
    base, n, k, b = PRESETS[name]
    d = dict(base)
    d["len_min"] = d["len_min"] * scale
    d["len_max"] = d["len_max"] * scale
    if scale < 1.0:
        d["mobile_min"] = max(200, int(d["mobile_min"] * scale))
        d["mobile_max"] = max(400, int(d["mobile_max"] * scale))
    d.update(override)
    return make_params(seed=seed, **d), n, k, b


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.cdbg_synth_write_fasta.argtypes = [
            ctypes.POINTER(SynthParams), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
            ctypes.c_int, ctypes.c_uint32, ctypes.c_char_p]
        _lib.cdbg_synth_write_fasta.restype = ctypes.c_int
        _lib.cdbg_synth_collection.argtypes = [
            ctypes.POINTER(SynthParams), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
            ctypes.POINTER(ctypes.c_uint64)]
        _lib.cdbg_synth_collection.restype = ctypes.c_int64
    return _lib


def write_fasta(params, num_genomes, out_dir, gzip_level=0, threads=None, g0=0):
    """Write genomes g0..g0+num_genomes-1 as FASTA; returns the filenames-list path."""
    os.makedirs(out_dir, exist_ok=True)
    listp = os.path.join(out_dir, "filenames.txt")
    rc = lib().cdbg_synth_write_fasta(ctypes.byref(params), g0, g0 + num_genomes,
                                      out_dir.encode(), gzip_level, threads or os.cpu_count(),
                                      listp.encode())
    if rc != 0:
        raise RuntimeError("cdbg_synth_write_fasta failed (%d)" % rc)
    return listp


def collection(params, num_genomes, threads=None, g0=0):
    """Genomes as (ascii bytes as numpy uint8, contig lengths u64, contigs per genome u32)."""
    import numpy as np
    tot = ctypes.c_uint64(0)
    n = lib().cdbg_synth_collection(ctypes.byref(params), g0, g0 + num_genomes,
                                    threads or os.cpu_count(), None, 0, None, 0, None,
                                    ctypes.byref(tot))
    if n < 0:
        raise RuntimeError("cdbg_synth_collection failed")
    seq = np.empty(n, dtype=np.uint8)
    lens = np.empty(tot.value, dtype=np.uint64)
    per = np.empty(num_genomes, dtype=np.uint32)
    n2 = lib().cdbg_synth_collection(ctypes.byref(params), g0, g0 + num_genomes,
                                     threads or os.cpu_count(), seq.ctypes.data, n,
                                     lens.ctypes.data, tot.value, per.ctypes.data,
                                     ctypes.byref(tot))
    if n2 != n:
        raise RuntimeError("cdbg_synth_collection size mismatch")
    return seq, lens, per
