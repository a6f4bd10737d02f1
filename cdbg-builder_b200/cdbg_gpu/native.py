"""ctypes binding of libcdbg_gpu.so (include/cdbg_gpu.h).

Mirrors the reference's phase entry points:

* ``Engine.phase1``  <- ``cdbg::ingest_bucketed`` + ``bucket_writer::close``
  (phase1_bucket_write/bucket_ingester.hpp:183, bucket_io.hpp:389)
* ``Engine.phase2``  <- ``cdbg::process_buckets``
  (phase2_bucket_process/bucket_walker.hpp:608)
* ``Engine.build``   <- both, in memory (builder.hpp:180 + :269)

Errors raise ``RuntimeError`` with the library's message, as the reference
throws ``std::runtime_error``.  There is no fallback: if the library is
missing or no CUDA device is present the calls fail.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libcdbg_gpu.so")

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)


class SeqBatch(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_void_p), ("seq_bytes", ctypes.c_uint64),
                ("seq_off", ctypes.c_void_p), ("seq_color", ctypes.c_void_p),
                ("num_seqs", ctypes.c_uint32), ("on_device", ctypes.c_int32)]


class Phase1Args(ctypes.Structure):
    _fields_ = [("files", ctypes.POINTER(ctypes.c_char_p)), ("num_files", ctypes.c_uint32),
                ("k", ctypes.c_uint32), ("m", ctypes.c_uint32), ("num_buckets", ctypes.c_uint32),
                ("tmp_dir", ctypes.c_char_p), ("host_threads", ctypes.c_uint32),
                ("chunk_bytes", ctypes.c_uint64), ("bucket_unc_bytes", c_u64p), ("first_color", ctypes.c_uint32)]


class Phase1Stats(ctypes.Structure):
    _fields_ = [("input_bytes", ctypes.c_uint64), ("seq_bytes", ctypes.c_uint64),
                ("n_kmers", ctypes.c_uint64), ("n_supers", ctypes.c_uint64),
                ("n_records", ctypes.c_uint64), ("unc_bytes", ctypes.c_uint64),
                ("comp_bytes", ctypes.c_uint64), ("seconds_total", ctypes.c_double),
                ("seconds_device", ctypes.c_double)]


CLASS_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, c_u32p, ctypes.c_uint64)


class Phase2Args(ctypes.Structure):
    _fields_ = [("tmp_dir", ctypes.c_char_p), ("num_buckets", ctypes.c_uint32),
                ("k", ctypes.c_uint32), ("num_colors", ctypes.c_uint32),
                ("frag_path", ctypes.c_char_p), ("color_sets_path", ctypes.c_char_p),
                ("on_class", CLASS_CB), ("ctx", ctypes.c_void_p),
                ("delete_consumed", ctypes.c_int32), ("host_threads", ctypes.c_uint32),
                ("batch_occ", ctypes.c_uint64), ("pass_bytes", ctypes.c_uint64)]


class Phase2Stats(ctypes.Structure):
    _fields_ = [("n_records", ctypes.c_uint64), ("n_kmers", ctypes.c_uint64),
                ("n_distinct", ctypes.c_uint64), ("n_fragments", ctypes.c_uint64),
                ("total_seq_bytes", ctypes.c_uint64), ("n_color_sets", ctypes.c_uint64),
                ("total_integers", ctypes.c_uint64), ("color_bits", ctypes.c_uint64),
                ("seconds_total", ctypes.c_double), ("seconds_device", ctypes.c_double),
                ("n_passes", ctypes.c_uint64)]


class BuildParams(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("m", ctypes.c_uint32), ("num_buckets", ctypes.c_uint32),
                ("num_colors", ctypes.c_uint32), ("batch_occ", ctypes.c_uint64),
                ("outputs_to_host", ctypes.c_int32), ("bucket_lo", ctypes.c_uint32),
                ("bucket_hi", ctypes.c_uint32)]


class BuildFilesArgs(ctypes.Structure):
    _fields_ = [("files", ctypes.POINTER(ctypes.c_char_p)), ("num_files", ctypes.c_uint32),
                ("k", ctypes.c_uint32), ("m", ctypes.c_uint32), ("num_buckets", ctypes.c_uint32),
                ("host_threads", ctypes.c_uint32), ("batch_occ", ctypes.c_uint64),
                ("frag_path", ctypes.c_char_p), ("color_sets_path", ctypes.c_char_p),
                ("stitch_dir", ctypes.c_char_p), ("stitch_closed_path", ctypes.c_char_p),
                ("stitch_buckets", ctypes.c_uint32), ("stitch_kmer_bits", ctypes.c_uint32)]


class BuildResult(ctypes.Structure):
    _fields_ = [("frag_bytes", ctypes.c_void_p), ("frag_nbytes", ctypes.c_uint64),
                ("class_words", ctypes.c_void_p), ("class_bits", ctypes.c_uint64),
                ("class_offsets", ctypes.c_void_p), ("n_color_sets", ctypes.c_uint64),
                ("total_integers", ctypes.c_uint64), ("n_kmers", ctypes.c_uint64),
                ("n_supers", ctypes.c_uint64), ("n_records", ctypes.c_uint64),
                ("n_occ", ctypes.c_uint64), ("n_distinct", ctypes.c_uint64),
                ("n_fragments", ctypes.c_uint64), ("total_seq_bytes", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("n_bases", ctypes.c_uint64),
                ("ms_phase1", ctypes.c_double), ("ms_phase2", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("ms_outputs", ctypes.c_double), ("ms_seed", ctypes.c_double),
                ("seed_routed", ctypes.c_uint64), ("seed_closed_unitigs", ctypes.c_uint64)]


class MergedRecords(ctypes.Structure):
    _fields_ = [("bytes", ctypes.c_void_p), ("nbytes", ctypes.c_uint64), ("bucket_off", ctypes.c_void_p),
                ("handle", ctypes.c_void_p)]


class SeedArgs(ctypes.Structure):
    _fields_ = [("frags", ctypes.c_void_p), ("frag_nbytes", ctypes.c_uint64), ("k", ctypes.c_uint32),
                ("num_buckets", ctypes.c_uint32), ("kmer_bits", ctypes.c_uint32),
                ("host_threads", ctypes.c_uint32), ("chunk_bytes", ctypes.c_uint64),
                ("round_dir", ctypes.c_char_p), ("closed_path", ctypes.c_char_p)]


class SeedStats(ctypes.Structure):
    _fields_ = [("fragments", ctypes.c_uint64), ("routed", ctypes.c_uint64),
                ("closed_fragments", ctypes.c_uint64), ("closed_unitigs", ctypes.c_uint64),
                ("routed_frag_bytes", ctypes.c_uint64), ("round0_bytes", ctypes.c_uint64), ("round0_file_bytes", ctypes.c_uint64),
                ("closed", ctypes.c_void_p), ("closed_nbytes", ctypes.c_uint64), ("n_passes", ctypes.c_uint64),
                ("ms_scan", ctypes.c_double), ("ms_device", ctypes.c_double), ("ms_files", ctypes.c_double),
                ("ms_total", ctypes.c_double)]


class Merged(ctypes.Structure):
    _fields_ = [("frag_bytes", ctypes.c_void_p), ("frag_nbytes", ctypes.c_uint64),
                ("class_words", ctypes.c_void_p), ("class_bits", ctypes.c_uint64),
                ("class_offsets", ctypes.c_void_p), ("n_color_sets", ctypes.c_uint64),
                ("handle", ctypes.c_void_p)]


class Tuning(ctypes.Structure):
    _fields_ = [("batch_occ", ctypes.c_uint64), ("minimizer_tile", ctypes.c_uint32),
                ("heavy_colors", ctypes.c_uint32), ("table_slots_q", ctypes.c_uint32),
                ("union_lists", ctypes.c_uint32), ("table_group_mb", ctypes.c_uint32),
                ("radix_bits", ctypes.c_uint32), ("gpu_inflate", ctypes.c_uint32)]


class ServerParams(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_uint32), ("hbm_budget", ctypes.c_uint64),
                ("bytes_per_base", ctypes.c_double), ("floor_bytes", ctypes.c_uint64)]


class RequestResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("error", ctypes.c_char_p),
                ("frag_bytes", ctypes.c_void_p), ("frag_nbytes", ctypes.c_uint64),
                ("class_words", ctypes.c_void_p), ("class_bits", ctypes.c_uint64),
                ("class_offsets", ctypes.c_void_p), ("n_color_sets", ctypes.c_uint64),
                ("total_integers", ctypes.c_uint64), ("n_kmers", ctypes.c_uint64),
                ("n_distinct", ctypes.c_uint64), ("n_fragments", ctypes.c_uint64),
                ("need_bytes", ctypes.c_uint64), ("grant_bytes", ctypes.c_uint64),
                ("t_submit", ctypes.c_double), ("t_start", ctypes.c_double), ("t_done", ctypes.c_double),
                ("ms_device", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("waiting", ctypes.c_uint64),
                ("running", ctypes.c_uint32), ("peak_running", ctypes.c_uint32),
                ("reserved_bytes", ctypes.c_uint64), ("peak_reserved_bytes", ctypes.c_uint64),
                ("clock_s", ctypes.c_double)]


# symbol -> (restype, argtypes); the header's complete list
SIGNATURES = {
    "cdbg_engine_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "cdbg_engine_destroy": (None, [ctypes.c_void_p]),
    "cdbg_last_error": (ctypes.c_char_p, []),
    "cdbg_gpu_version": (ctypes.c_int, []),
    "cdbg_engine_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cdbg_launch_count": (ctypes.c_uint64, []),
    "cdbg_engine_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "cdbg_engine_kernel_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64,
                                                ctypes.POINTER(ctypes.c_double), ctypes.c_uint32]),
    "cdbg_engine_kernel_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64,
                                                ctypes.POINTER(ctypes.c_double), c_u64p, ctypes.c_uint32]),
    "cdbg_gpu_supers_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_uint64, c_u64p,
                                               ctypes.c_void_p]),
    "cdbg_engine_copy_out": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_uint64]),
    "cdbg_read_sequences": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_uint32,
                                           ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(SeqBatch)]),
    "cdbg_free_sequences": (None, [ctypes.POINTER(SeqBatch)]),
    "cdbg_gpu_phase1": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Phase1Args),
                                       ctypes.POINTER(Phase1Stats)]),
    "cdbg_gpu_dump_supers": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SeqBatch),
                                            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_char_p, c_u64p]),
    "cdbg_gpu_sort_pairs_u64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_uint64]),
    "cdbg_gpu_gunzip": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), c_u64p, ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_void_p), c_u64p, c_u64p,
                                       ctypes.POINTER(ctypes.c_uint32)]),
    "cdbg_gpu_phase2": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Phase2Args),
                                       ctypes.POINTER(Phase2Stats)]),
    "cdbg_gpu_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SeqBatch),
                                      ctypes.POINTER(BuildParams), ctypes.POINTER(BuildResult)]),
    "cdbg_gpu_build_files": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BuildFilesArgs),
                                            ctypes.POINTER(BuildResult)]),
    "cdbg_gpu_stitch_seed": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SeedArgs),
                                            ctypes.POINTER(SeedStats)]),
    "cdbg_frag_record_offsets": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, c_u64p,
                                                ctypes.c_uint64, c_u64p]),
    "cdbg_engine_set_memory_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "cdbg_engine_memory": (ctypes.c_int, [ctypes.c_void_p, c_u64p, c_u64p]),
    "cdbg_engine_trim": (ctypes.c_int, [ctypes.c_void_p]),
    "cdbg_engine_record_bytes": (ctypes.c_int, [ctypes.c_void_p, c_u64p]),
    "cdbg_engine_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    "cdbg_engine_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    "cdbg_engine_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SeqBatch), ctypes.POINTER(BuildParams),
                                            ctypes.c_uint32, ctypes.POINTER(Tuning),
                                            ctypes.POINTER(ctypes.c_double)]),
    "cdbg_server_create": (ctypes.c_int, [ctypes.POINTER(ServerParams), ctypes.POINTER(ctypes.c_void_p)]),
    "cdbg_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SeqBatch),
                                          ctypes.POINTER(BuildParams), c_u64p]),
    "cdbg_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(RequestResult)]),
    "cdbg_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "cdbg_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "cdbg_server_destroy": (None, [ctypes.c_void_p]),
    "cdbg_server_last_error": (ctypes.c_char_p, []),
    "cdbg_merge_shards": (ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p), c_u64p,
                                         ctypes.POINTER(ctypes.c_void_p), c_u64p,
                                         ctypes.POINTER(ctypes.c_void_p), c_u64p, ctypes.c_void_p]),
    "cdbg_merged_free": (None, [ctypes.c_void_p]),
    "cdbg_merge_bucket_records": (ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p),
                                                 ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint32, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.POINTER(MergedRecords)]),
    "cdbg_merged_records_free": (None, [ctypes.POINTER(MergedRecords)]),
    "cdbg_class_strings": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "cdbg_frag_remap_classes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                               ctypes.c_uint64]),
    "cdbg_merge_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """Load libcdbg_gpu.so (raises OSError when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libcdbg_gpu.so not built: run cdbg-builder_b200/build.py (%s)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().cdbg_last_error().decode(errors="replace"))


def best_m(k):
    """compute_best_m (phase1_bucket_write/minimizer.hpp:65-73)."""
    if k <= 13:
        return (k // 2) if (k // 2 > k - 4) else (k - 4 if k > 4 else 1)
    for lim, m in ((15, 9), (21, 10), (30, 11), (37, 12), (42, 13), (64, 14)):
        if k <= lim:
            return m
    return (k + 2) // 4


def host_batch(seqs, colors):
    """SeqBatch over host arrays built from Python byte strings (keeps refs alive)."""
    data = b"".join(seqs)
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    if seqs:
        off[1:] = np.cumsum([len(s) for s in seqs])
    col = np.asarray(colors, dtype=np.uint32)
    buf = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, dtype=np.uint8)
    b = SeqBatch(buf.ctypes.data, len(data), off.ctypes.data, col.ctypes.data, len(seqs), 0)
    b._keep = (buf, off, col)
    return b


def array_batch(seq_u8, seq_off_u64, colors_u32, on_device=False):
    """SeqBatch over numpy arrays (host) or raw device pointers (on_device=True)."""
    if on_device:
        b = SeqBatch(seq_u8[0], seq_u8[1], seq_off_u64, colors_u32[0], colors_u32[1], 1)
        return b
    b = SeqBatch(seq_u8.ctypes.data, seq_u8.nbytes, seq_off_u64.ctypes.data,
                 colors_u32.ctypes.data, len(colors_u32), 0)
    b._keep = (seq_u8, seq_off_u64, colors_u32)
    return b


class HostSequences:
    """Sequences of FASTA/FASTQ(.gz) files read by the library's host reader
    (kseq record rules); `.batch` is the SeqBatch to pass to Engine calls."""

    def __init__(self, files, first_color=0, host_threads=0):
        arr = (ctypes.c_char_p * len(files))(*[f.encode() for f in files])
        self.batch = SeqBatch()
        _check(lib().cdbg_read_sequences(arr, len(files), first_color, host_threads,
                                         ctypes.byref(self.batch)))

    def close(self):
        if self.batch.seq_off:
            lib().cdbg_free_sequences(ctypes.byref(self.batch))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def seq_bytes(self):
        return ctypes.string_at(self.batch.seq, self.batch.seq_bytes)

    def offsets(self):
        return np.ctypeslib.as_array(ctypes.cast(self.batch.seq_off, c_u64p),
                                     shape=(self.batch.num_seqs + 1,)).copy()

    def colors(self):
        if self.batch.num_seqs == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(ctypes.cast(self.batch.seq_color, c_u32p),
                                     shape=(self.batch.num_seqs,)).copy()


class Engine:
    """One CUDA device, one stream, a cached device arena."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        _check(lib().cdbg_engine_create(device, ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib().cdbg_engine_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_memory_limit(self, nbytes):
        """Cap the device memory of this engine's calls (0 = none)."""
        _check(lib().cdbg_engine_set_memory_limit(self._h, nbytes))

    def memory(self):
        """(bytes held now, peak since the previous call)."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().cdbg_engine_memory(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_tuning(self, batch_occ=0, minimizer_tile=0, heavy_colors=0, table_slots_q=0, union_lists=0,
                   table_group_mb=0, radix_bits=0, gpu_inflate=0):
        _check(lib().cdbg_engine_set_tuning(self._h, ctypes.byref(Tuning(batch_occ, minimizer_tile, heavy_colors,
                                                                         table_slots_q, union_lists,
                                                                         table_group_mb, radix_bits,
                                                                         gpu_inflate))))

    def tuning(self):
        t = Tuning()
        _check(lib().cdbg_engine_get_tuning(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def autotune(self, batch, k, num_buckets, num_colors, m=0, rounds=1):
        """Search the performance knobs on `batch`; the engine keeps the best.
        Returns (tuning dict, best device ms)."""
        p = BuildParams(k, m, num_buckets, num_colors, 0, 0)
        t, ms = Tuning(), ctypes.c_double()
        _check(lib().cdbg_engine_autotune(self._h, ctypes.byref(batch), ctypes.byref(p), rounds, ctypes.byref(t),
                                          ctypes.byref(ms)))
        return {k2: getattr(t, k2) for k2, _ in Tuning._fields_}, ms.value

    def record_bytes(self):
        """Serialized bucket-record bytes of the last build()."""
        v = ctypes.c_uint64()
        _check(lib().cdbg_engine_record_bytes(self._h, ctypes.byref(v)))
        return v.value

    def trim(self):
        """Return cached device memory to the device pool."""
        _check(lib().cdbg_engine_trim(self._h))

    def set_stream(self, stream_handle):
        """Run on a caller-owned cudaStream_t (int handle, e.g. torch's
        Stream.cuda_stream); None restores the engine's own stream."""
        _check(lib().cdbg_engine_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def profile(self, enable=True):
        _check(lib().cdbg_engine_profile(self._h, 1 if enable else 0))

    def kernel_stats(self):
        """{kernel name: (total ms, launches)} collected while profiling."""
        cap = 256
        names = ctypes.create_string_buffer(64 * cap)
        ms = (ctypes.c_double * cap)()
        ln = (ctypes.c_uint64 * cap)()
        n = lib().cdbg_engine_kernel_stats(self._h, names, len(names), ms, ln, cap)
        if n < 0:
            raise RuntimeError("kernel stats failed")
        keys = names.raw.split(b"\0")[:min(n, cap)]
        return {keys[i].decode(): (ms[i], ln[i]) for i in range(min(n, cap))}

    def kernel_bytes(self):
        """{kernel name: algorithmic bytes} declared by the launch sites while profiling."""
        cap = 256
        names = ctypes.create_string_buffer(64 * cap)
        b = (ctypes.c_double * cap)()
        n = lib().cdbg_engine_kernel_bytes(self._h, names, len(names), b, cap)
        if n < 0:
            raise RuntimeError("kernel bytes failed")
        keys = names.raw.split(b"\0")[:min(n, cap)]
        return {keys[i].decode(): b[i] for i in range(min(n, cap))}

    def sort_pairs_u64(self, keys_ptr, vals_ptr, n):
        """Stable in-place sort of n device (u64 key, u32 value) pairs by key."""
        _check(lib().cdbg_gpu_sort_pairs_u64(self._h, keys_ptr, vals_ptr, n))

    def gunzip(self, streams, caps):
        """Device gzip decoder on byte strings `streams` (out_caps `caps`):
        [(status, bytes)] per stream."""
        n = len(streams)
        bufs = [ctypes.create_string_buffer(max(int(c), 1)) for c in caps]
        keep = [ctypes.create_string_buffer(bytes(x), len(x)) if len(x) else ctypes.create_string_buffer(1)
                for x in streams]
        sp = (ctypes.c_void_p * max(n, 1))(*[ctypes.cast(b, ctypes.c_void_p) for b in keep])
        op = (ctypes.c_void_p * max(n, 1))(*[ctypes.cast(b, ctypes.c_void_p) for b in bufs])
        lens = np.array([len(x) for x in streams] + [0], dtype=np.uint64)
        capa = np.array(list(caps) + [0], dtype=np.uint64)
        olen = np.zeros(n + 1, dtype=np.uint64)
        st = (ctypes.c_uint32 * max(n, 1))()
        _check(lib().cdbg_gpu_gunzip(self._h, sp, lens.ctypes.data_as(c_u64p), n, op, capa.ctypes.data_as(c_u64p),
                                     olen.ctypes.data_as(c_u64p), st))
        return [(int(st[i]), bufs[i].raw[:int(olen[i])] if st[i] == 0 else b"") for i in range(n)]

    def dump_supers(self, batch, k, m, num_buckets, path):
        n = ctypes.c_uint64()
        _check(lib().cdbg_gpu_dump_supers(self._h, ctypes.byref(batch), k, m, num_buckets,
                                          path.encode(), ctypes.byref(n)))
        return n.value

    def phase1(self, files, k, num_buckets, tmp_dir, m=0, host_threads=0, chunk_bytes=0, first_color=0):
        arr = (ctypes.c_char_p * len(files))(*[f.encode() for f in files])
        unc = np.zeros(num_buckets, dtype=np.uint64)
        a = Phase1Args(arr, len(files), k, m, num_buckets, tmp_dir.encode(), host_threads,
                       chunk_bytes, unc.ctypes.data_as(c_u64p), first_color)
        s = Phase1Stats()
        _check(lib().cdbg_gpu_phase1(self._h, ctypes.byref(a), ctypes.byref(s)))
        return s, unc

    def phase2(self, tmp_dir, num_buckets, k, num_colors, frag_path, color_sets_path=None,
               on_class=None, delete_consumed=False, host_threads=0, batch_occ=0, pass_bytes=0):
        cb = CLASS_CB(0)
        if on_class is not None:
            def _cb(ctx, p, n):
                on_class(np.ctypeslib.as_array(p, shape=(n,)).copy() if n else
                         np.zeros(0, dtype=np.uint32))
            cb = CLASS_CB(_cb)
        a = Phase2Args(tmp_dir.encode(), num_buckets, k, num_colors, frag_path.encode(),
                       color_sets_path.encode() if color_sets_path else None, cb, None,
                       1 if delete_consumed else 0, host_threads, batch_occ, pass_bytes)
        s = Phase2Stats()
        _check(lib().cdbg_gpu_phase2(self._h, ctypes.byref(a), ctypes.byref(s)))
        return s

    def copy_out(self, device_ptr, nbytes):
        """Host bytes of a device-resident build output."""
        buf = ctypes.create_string_buffer(max(1, nbytes))
        _check(lib().cdbg_engine_copy_out(self._h, ctypes.c_void_p(device_ptr), buf, nbytes))
        return buf.raw[:nbytes]

    def build_files(self, files, k, num_buckets, frag_path=None, color_sets_path=None, m=0, host_threads=0,
                    batch_occ=0, stitch_dir=None, stitch_closed_path=None, stitch_buckets=0, stitch_kmer_bits=0):
        """cdbg_gpu_build_files: files in, frag_unitigs.bin / .color_sets out
        (or, with no paths, outputs in host memory); with stitch_dir, also the
        stitch's round-0 files from the fragments in HBM."""
        arr = (ctypes.c_char_p * len(files))(*[f.encode() for f in files])
        enc = lambda x: x.encode() if x else None  # noqa: E731
        a = BuildFilesArgs(arr, len(files), k, m, num_buckets, host_threads, batch_occ, enc(frag_path),
                           enc(color_sets_path), enc(stitch_dir), enc(stitch_closed_path), stitch_buckets,
                           stitch_kmer_bits)
        r = BuildResult()
        _check(lib().cdbg_gpu_build_files(self._h, ctypes.byref(a), ctypes.byref(r)))
        return r

    def stitch_seed(self, frags, k, round_dir, num_buckets=1024, closed_path=None, kmer_bits=0, host_threads=0,
                    chunk_bytes=0):
        """cdbg_gpu_stitch_seed: round 0 of the stitch from frag_unitigs.bin
        bytes (bytes, a buffer, or (address, nbytes) of host memory).  Returns
        the stats as a dict; with no closed_path, 'closed' holds the closed
        unitigs' frag records."""
        if isinstance(frags, tuple):
            addr, n = frags
            keep = None
        else:
            keep = (ctypes.c_char * len(frags)).from_buffer_copy(frags) if len(frags) else None
            addr, n = (ctypes.addressof(keep) if keep is not None else None), len(frags)
        a = SeedArgs(addr, n, k, num_buckets, kmer_bits, host_threads, chunk_bytes, round_dir.encode(),
                     closed_path.encode() if closed_path else None)
        st = SeedStats()
        _check(lib().cdbg_gpu_stitch_seed(self._h, ctypes.byref(a), ctypes.byref(st)))
        out = {name: getattr(st, name) for name, _ in SeedStats._fields_ if name != "closed"}
        if not closed_path:
            out["closed"] = ctypes.string_at(st.closed, st.closed_nbytes) if st.closed_nbytes else b""
        return out

    def build(self, batch, k, num_buckets, num_colors, m=0, batch_occ=0, outputs_to_host=True, buckets=None):
        lo, hi = buckets if buckets else (0, 0)
        p = BuildParams(k, m, num_buckets, num_colors, batch_occ, 1 if outputs_to_host else 0, lo, hi)
        r = BuildResult()
        _check(lib().cdbg_gpu_build(self._h, ctypes.byref(batch), ctypes.byref(p), ctypes.byref(r)))
        return r


def frag_record_offsets(frags, host_threads=0):
    """Record offsets of frag_unitigs.bin bytes (numpy uint64, records + 1)."""
    import numpy as np
    buf = (ctypes.c_char * len(frags)).from_buffer_copy(frags) if len(frags) else None
    n = ctypes.c_uint64()
    _check(lib().cdbg_frag_record_offsets(buf, len(frags), host_threads, None, 0, ctypes.byref(n)))
    out = np.zeros(n.value + 1, dtype=np.uint64)
    _check(lib().cdbg_frag_record_offsets(buf, len(frags), host_threads,
                                          out.ctypes.data_as(c_u64p), len(out), ctypes.byref(n)))
    return out


def launch_count():
    """Kernel launches issued by libcdbg_gpu.so in this process."""
    return lib().cdbg_launch_count()


def result_frag_bytes(r):
    """Host copy of a BuildResult's frag bytes (outputs_to_host=True)."""
    return ctypes.string_at(r.frag_bytes, r.frag_nbytes) if r.frag_nbytes else b""


def result_class_words(r):
    n = (r.class_bits + 63) // 64
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.ctypeslib.as_array(ctypes.cast(r.class_words, c_u64p), shape=(n,)).copy()


def result_class_offsets(r):
    if r.n_color_sets == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.ctypeslib.as_array(ctypes.cast(r.class_offsets, c_u64p), shape=(r.n_color_sets,)).copy()


class Server:
    """Build server (include/cdbg_gpu.h cdbg_server_*): concurrent builds on
    one GPU under an HBM budget.  submit() returns a request id; wait()
    returns the finished request as a dict with its outputs (bytes, numpy
    words and offsets) and timings on the server's clock."""

    def __init__(self, device=0, slots=4, hbm_budget=150 << 30, bytes_per_base=0.0, floor_bytes=0):
        L = lib()
        p = ServerParams(device, slots, hbm_budget, bytes_per_base, floor_bytes)
        h = ctypes.c_void_p()
        if L.cdbg_server_create(ctypes.byref(p), ctypes.byref(h)) != 0:
            raise RuntimeError(L.cdbg_server_last_error().decode(errors="replace"))
        self.h = h
        self._keep = {}

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(lib().cdbg_server_last_error().decode(errors="replace"))

    def submit(self, batch, k, num_buckets, num_colors, m=0, batch_occ=0):
        p = BuildParams(k, m, num_buckets, num_colors, batch_occ, 1)
        rid = ctypes.c_uint64()
        self._check(lib().cdbg_server_submit(self.h, ctypes.byref(batch), ctypes.byref(p), ctypes.byref(rid)))
        self._keep[rid.value] = batch  # host buffers live until the request is done
        return rid.value

    def wait(self, rid, release=True, outputs=True):
        """Finished request `rid` as a dict; with outputs=False only counts and
        timings (no host copies of the outputs)."""
        r = RequestResult()
        self._check(lib().cdbg_server_wait(self.h, rid, ctypes.byref(r)))
        out = {k: getattr(r, k) for k, _ in RequestResult._fields_
               if k not in ("frag_bytes", "class_words", "class_offsets", "error")}
        out["error"] = r.error.decode(errors="replace") if r.error else ""
        if r.status == 0 and outputs:
            out["frag"] = ctypes.string_at(r.frag_bytes, r.frag_nbytes) if r.frag_nbytes else b""
            nw = (r.class_bits + 63) // 64
            out["words"] = np.ctypeslib.as_array(ctypes.cast(r.class_words, c_u64p), (nw,)).copy() \
                if nw else np.zeros(0, np.uint64)
            out["offsets"] = np.ctypeslib.as_array(ctypes.cast(r.class_offsets, c_u64p), (r.n_color_sets,)).copy() \
                if r.n_color_sets else np.zeros(0, np.uint64)
        if release:
            self._check(lib().cdbg_server_release(self.h, rid))
            self._keep.pop(rid, None)
        return out

    def stats(self):
        s = ServerStats()
        self._check(lib().cdbg_server_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().cdbg_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
