"""Benchmark: phase 1 + phase 2 k-mers/s on one B200 (or N replicas).

Workload (default): the pangenome configuration -- 1000 synthetic genomes of
~4.8 Mbp derived from one seeded ancestor (0.1-2% SNPs, 20 indels, one mobile
insert, 1-200 contigs), k = 31, m = 12, 4096 buckets.  A step is one full pass
of phase 1 + phase 2 over the whole collection (all k-mers), producing the
frag spill and the color classes.

  value     k-mers/s with the sequences already resident in HBM and the
            outputs left on the device (cdbg_gpu_build, on_device = 1); CUDA
            events on the stream the library launches on.
  e2e       the reference's inputs and outputs: the collection as gzip FASTA
            files on disk in, frag_unitigs.bin and .color_sets files out
            (cdbg_gpu_build_files: host inflate and parse overlapped with the
            upload and phase 1, phase 2 in HBM, outputs written); wall time
            of each call.
  e2e_host  pinned host sequences in, host outputs out (cdbg_gpu_build).

`--workload stitch-seed` times round 0 of the stitch instead
(cdbg_gpu_stitch_seed over the pangenome build's frag_unitigs.bin, round-0
files and closed unitigs written), in fragments/s, with the reference's own
seed (oracle/_ref/ref_seed) on the same file as its CPU baseline.

Max over ranks.  `--impl reference` times the reference's own phase 1 +
phase 2 (oracle/_ref/ref_phase12: the builder's ingest_bucketed, close and
process_buckets, built from the reference's sources) with all host cores on
bounded samples of the same collection: step i runs slice i mod 8 of every
genome.  With --gpus N each rank builds its own collection (independent
replicas, weak scaling).
"""
import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cdbg-builder_b200"))

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
REF_P12 = os.path.join(ROOT, "oracle", "_ref", "ref_phase12")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="pangenome")
    ap.add_argument("--genomes", type=int, default=0, help="override genome count (0 = workload's)")
    ap.add_argument("--genome-scale", type=float, default=1.0,
                    help="scale the workload's genome lengths (small cases for profiling; 1 = the workload)")
    ap.add_argument("--ref-slices", type=int, default=8,
                    help="reference CPU runs: 1/N of every genome per step (rotating over the N slices)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--check", action="store_true",
                    help="also check the benchmarked path's outputs on the reference arm's first sample "
                         "against the reference's own phase 2 (one thread), byte for byte")
    ap.add_argument("--e2e-dir", default="", help="directory for the e2e input/output files (default: temp)")
    ap.add_argument("--batch-occ", type=int, default=0)
    ap.add_argument("--table-slots-q", type=int, default=0,
                    help="k-mer table slots per 4 occurrences, 5..16 (0 = library default)")
    ap.add_argument("--tuning", default="", help='knobs of cdbg_tuning as JSON, e.g. {"minimizer_tile": 2048}')
    ap.add_argument("--autotune", action="store_true",
                    help="run the autotuner on the workload before timing (default for skewed)")
    ap.add_argument("--compare-plain", action="store_true",
                    help="also time one step of the plain one-bucket-per-batch path (default for skewed)")
    ap.add_argument("--out", default="")
    # serving workload
    ap.add_argument("--requests", type=int, default=512, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=30.0, help="serving: Poisson arrivals per second")
    ap.add_argument("--slots", default="1,2,3,4",
                    help="serving: concurrent builds; a list is swept and the best is reported")
    ap.add_argument("--no-plain", action="store_true", help="serving: skip the plain one-at-a-time run")
    ap.add_argument("--plain-requests", type=int, default=48,
                    help="serving: requests of the stream the plain one-at-a-time path serves")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--serving-buckets", type=int, default=1024)
    ap.add_argument("--seed-buckets", type=int, default=1024, help="stitch-seed: round-store buckets")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), \
        int(os.environ.get("WORLD_SIZE", "1"))


def max_over_ranks(v, world, device):
    """The largest per-rank value over all ranks (the slowest rank's time)."""
    return _reduce(v, world, device, "max")


def sum_over_ranks(v, world, device):
    """Per-rank counts summed over all ranks (units the whole job processed)."""
    return _reduce(v, world, device, "sum")


def _reduce(v, world, device, how):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if how == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def count_kmers(lens, k):
    import numpy as np
    l = lens.astype(np.int64)
    return int(np.maximum(l - k + 1, 0).sum())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                   "--format=csv,noheader,nounits", "-lms", "200"],
                                  stdout=self.f, stderr=subprocess.DEVNULL)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        d = json.load(open(PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- reference arm
def scratch_base(want_bytes=40 << 30):
    """Where both arms keep their input and output files: a RAM-backed file
    system when the host has one with room (the outputs of a step are several
    GB; written to a disk, steps back to back end up waiting on its write-back,
    which neither arm's own work decides), else the default temporary
    directory."""
    d = "/dev/shm"
    try:
        st = os.statvfs(d)
        if os.access(d, os.W_OK) and st.f_bavail * st.f_frsize >= want_bytes:
            return d
    except OSError:
        pass
    return None


def write_slice(seq, lens, per, s, nslices, k, out_dir, threads):
    """Slice s of nslices of every genome of a collection (bases [s*T/S,
    (s+1)*T/S) of each genome's concatenated contigs, contig boundaries kept),
    one gzip FASTA file per genome (= one color), like the workload's inputs.
    Returns (filenames list path, k-mers in the slice)."""
    import zlib
    from concurrent.futures import ThreadPoolExecutor
    import numpy as np
    os.makedirs(out_dir, exist_ok=True)
    lens = lens.astype(np.int64)
    ends = np.cumsum(lens)
    g_first = np.concatenate(([0], np.cumsum(per)))  # first contig of each genome
    contig_start = ends - lens
    names = []
    kmers = [0] * len(per)

    def one(g):
        c0, c1 = int(g_first[g]), int(g_first[g + 1])
        gs, ge = int(contig_start[c0]), int(ends[c1 - 1])
        T = ge - gs
        a, b = gs + T * s // nslices, gs + T * (s + 1) // nslices
        parts, km = [], 0
        for c in range(c0, c1):
            x, y = max(a, int(contig_start[c])), min(b, int(ends[c]))
            if y > x:
                parts.append(b">g%d_%d\n" % (g, c) + seq[x:y].tobytes() + b"\n")
                km += max(y - x - k + 1, 0)
        path = os.path.join(out_dir, "g%d.fa.gz" % g)
        co = zlib.compressobj(1, zlib.DEFLATED, 31)
        with open(path, "wb") as f:
            f.write(co.compress(b"".join(parts)))
            f.write(co.flush())
        kmers[g] = km
        return path

    with ThreadPoolExecutor(max_workers=threads) as ex:
        names = list(ex.map(one, range(len(per))))
    lst = os.path.join(out_dir, "filenames.txt")
    with open(lst, "w") as f:
        f.write("".join(n + "\n" for n in names))
    return lst, sum(kmers)


def run_ref_phase12(filelist, k, B, threads, workdir):
    """The reference's own phase 1 + phase 2 (oracle/_ref/ref_phase12: the
    builder's ingest_bucketed, close and process_buckets, nothing after) over
    the files; returns (seconds of the whole span, detail)."""
    tmp = os.path.join(workdir, "tmp")
    out = os.path.join(workdir, "out")
    shutil.rmtree(tmp, ignore_errors=True)
    shutil.rmtree(out, ignore_errors=True)
    binp = REF_P12 + ("-largek" if k > 31 else "")
    r = subprocess.run([binp, filelist, str(k), "0", str(B), str(threads), tmp, out], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("reference phase 1 + 2 failed: " + r.stderr[-500:])
    t = float(re.search(r"phase12_seconds=([0-9.eE+-]+)", r.stdout).group(1))
    t1 = float(re.search(r"\[bucket-write\] ([0-9.eE+-]+) s", r.stdout).group(1))
    t2 = float(re.search(r"\[bucket-process\] ([0-9.eE+-]+) s", r.stdout).group(1))
    shutil.rmtree(tmp, ignore_errors=True)
    shutil.rmtree(out, ignore_errors=True)
    return t, {"phase12_s": t, "bucket_write_s": t1, "bucket_process_s": t2}


class ReferenceSample:
    """Bounded samples of the benchmark's own collection for the reference's
    CPU build: the same seeded genomes as the GPU arm's (rank 0), cut into
    `nslices` slices of every genome, so a sample keeps every color and the
    collection's divergence structure; step i runs slice i mod nslices, so
    consecutive steps cover the whole collection."""

    def __init__(self, workload, n_genomes, nslices, threads, seed=1, scale=1.0):
        from cdbg_gpu import synth
        p, _, self.k, blog2 = synth.preset(workload, seed=seed, scale=scale)
        self.B = 1 << blog2
        self.n, self.S, self.threads = n_genomes, nslices, threads
        self.seq, self.lens, self.per = synth.collection(p, n_genomes)
        self.work = tempfile.mkdtemp(prefix="cdbg_ref_", dir=scratch_base())
        self.slices = {}

    def slice(self, s):
        s %= self.S
        if s not in self.slices:
            self.slices[s] = write_slice(self.seq, self.lens, self.per, s, self.S, self.k,
                                         os.path.join(self.work, "s%d" % s), self.threads)
        return self.slices[s]

    def run(self, s):
        lst, kmers = self.slice(s)
        t, det = run_ref_phase12(lst, self.k, self.B, self.threads, os.path.join(self.work, "run"))
        return kmers, t, det

    def describe(self, kmers):
        return ("slice i mod %d (1/%d of every one of the %d genomes, gzip FASTA) per step, ~%d k-mers; "
                "reference ingest_bucketed + close + process_buckets with -t %d, -b %d, files in %s" % (
                    self.S, self.S, self.n, kmers, self.threads, self.B.bit_length() - 1,
                    os.path.dirname(self.work)))

    def close(self):
        shutil.rmtree(self.work, ignore_errors=True)


def workload_name(n_genomes, k, B, workload="pangenome", scale=1.0):
    from cdbg_gpu.native import best_m
    shape = {
        "pangenome": "%d genomes x 4.8 Mbp (0.1-2%% SNPs, 1-200 contigs)",
        "small": "%d genomes x 5.0 Mbp (0.5%% SNPs, 20 indels, 1-3 contigs)",
        "largek": "%d genomes x 4.8 Mbp + 2%% tandem repeats + 200 shared 1-5 kbp repeats each",
        "skewed": "%d genomes x 1-6 Mbp log-uniform, 10%% homopolymer/dinucleotide runs",
    }.get(workload, "%d genomes")
    name = "%s: %s, k=%d, m=%d, %d buckets" % (workload, shape % n_genomes, k, best_m(k), B)
    return name if scale == 1.0 else name + ", genome lengths x%g" % scale


def workload_config(workload, n_genomes, k, B, seq_bytes, scale=1.0):
    """The `config` both arms print (identical, so the lines compare)."""
    from cdbg_gpu.native import best_m
    return {"workload": workload_name(n_genomes, k, B, workload, scale), "genomes": n_genomes, "k": k, "m": best_m(k),
            "buckets": B,
            "l2": ("inputs (%.1f GB) larger than L2" % (seq_bytes / 1e9)) if seq_bytes > 126e6 else
                  ("inputs (%.0f MB) smaller than L2, not flushed between steps" % (seq_bytes / 1e6))}


def reference_arm(a):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    if not os.path.exists(REF_P12):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_phase12 not built"}))
        return 0
    from cdbg_gpu import synth
    threads = os.cpu_count() or 1
    _, n_genomes, k, blog2 = synth.preset(a.workload)
    if a.genomes:
        n_genomes = a.genomes
    R = ReferenceSample(a.workload, n_genomes, a.ref_slices, threads, scale=a.genome_scale)
    try:
        i = 0
        for _ in range(a.warmup):
            R.run(i)
            i += 1
        km_tot, s_tot, secs, det = 0, 0.0, [], None
        for _ in range(a.steps):
            km, s, det = R.run(i)
            i += 1
            km_tot += km
            s_tot += s
            secs.append(s)
        sample = R.describe(km_tot // max(a.steps, 1))
        cfg = workload_config(a.workload, n_genomes, k, R.B, R.seq.nbytes, a.genome_scale)
    finally:
        R.close()
    v = km_tot / s_tot
    line = {"impl": "reference", "metric": "phase1+2 k-mers/s", "value": v, "unit": "k-mers/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000 * s_tot / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64" if k <= 31 else "u128", "data": "synthetic",
            "config": cfg, "sample": sample,
            "cpu_baseline": {"value": v, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                             "sample": sample, "last_step": det},
            "e2e": {"value": v, "unit": "k-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm
def main_gpu(a):
    import numpy as np
    import torch
    from cdbg_gpu import native, synth

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    p, n_genomes, k, blog2 = synth.preset(a.workload, seed=1 + rank, scale=a.genome_scale)
    if a.genomes:
        n_genomes = a.genomes
    B = 1 << blog2
    t0 = time.time()
    seq, lens, per = synth.collection(p, n_genomes)
    gen_s = time.time() - t0
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    colors = np.repeat(np.arange(n_genomes, dtype=np.uint32), per)
    kmers = count_kmers(lens, k)

    # host (pinned) and device copies of the inputs
    h_seq = torch.from_numpy(seq).pin_memory()
    h_off = torch.from_numpy(off.view(np.int64)).pin_memory()
    h_col = torch.from_numpy(colors.view(np.int32)).pin_memory()
    d_seq = h_seq.to("cuda")
    d_off = h_off.to("cuda")
    d_col = h_col.to("cuda")
    torch.cuda.synchronize()
    dev_batch = native.SeqBatch(d_seq.data_ptr(), seq.nbytes, d_off.data_ptr(), d_col.data_ptr(),
                                len(colors), 1)
    host_batch = native.SeqBatch(h_seq.data_ptr(), seq.nbytes, h_off.data_ptr(), h_col.data_ptr(),
                                 len(colors), 0)

    stream = torch.cuda.Stream()
    eng = native.Engine(local)
    eng.set_stream(stream.cuda_stream)

    def step(batch, to_host, batch_occ=None):
        return eng.build(batch, k, B, n_genomes, batch_occ=a.batch_occ if batch_occ is None else batch_occ,
                         outputs_to_host=to_host)

    skewed = a.workload == "skewed"
    tuned = None
    if a.table_slots_q or a.tuning:
        knobs = json.loads(a.tuning) if a.tuning else {}
        if a.table_slots_q:
            knobs["table_slots_q"] = a.table_slots_q
        eng.set_tuning(**knobs)
    if a.autotune or skewed:
        t0 = time.time()
        tcfg, tms = eng.autotune(dev_batch, k, B, n_genomes)
        tuned = {"tuning": tcfg, "best_ms": tms, "seconds": time.time() - t0}

    for _ in range(a.warmup):
        r = step(dev_batch, False)
    torch.cuda.synchronize()

    # ---- value: device-resident inputs
    clk = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clk.start()
    l0 = native.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    res = []
    for _ in range(a.steps):
        res.append(step(dev_batch, False))
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = native.launch_count() - l0
    clocks = clk.stop()
    barrier()
    ms = ev0.elapsed_time(ev1) / a.steps
    rec_bytes = eng.record_bytes()  # of the last timed build, counted outside the timed region
    # per-kernel CUDA-event times on the launching stream, from a second pass of
    # the same K steps (its per-kernel events cost the host some enqueue time,
    # so `value` comes from the pass above, which has none)
    eng.profile(True)
    torch.cuda.synchronize()
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(a.steps):
        step(dev_batch, False)
    k1.record(stream)
    torch.cuda.synchronize()
    kms = k0.elapsed_time(k1) / a.steps
    kstats = eng.kernel_stats()
    kbytes = eng.kernel_bytes()
    eng.profile(False)
    ms = max_over_ranks(ms, world, "cuda")
    job_kmers = sum_over_ranks(kmers, world, "cuda")  # every rank builds its own seeded collection
    r = res[-1]
    value = job_kmers / (ms / 1000.0)

    # ---- e2e: the reference's inputs and outputs -- the collection as gzip
    # FASTA files on disk in, frag_unitigs.bin and .color_sets files out --
    # through cdbg_gpu_build_files (host inflate/parse overlapped with the
    # upload and phase 1, phase 2 in HBM, device Elias-Fano finalize, file
    # writes); wall time of each call, max over ranks
    e2e = None
    e2e_host = None
    if not a.no_e2e:
        fdir = tempfile.mkdtemp(prefix="cdbg_e2e_", dir=a.e2e_dir or scratch_base())
        try:
            lst = synth.write_fasta(p, n_genomes, os.path.join(fdir, "in"), gzip_level=1)
            files = [l.strip() for l in open(lst) if l.strip()]
            gz_bytes = sum(os.path.getsize(f) for f in files)
            frag_p, cs_p = os.path.join(fdir, "frag_unitigs.bin"), os.path.join(fdir, "out.color_sets")
            for _ in range(max(1, min(a.warmup, 2))):
                eng.build_files(files, k, B, frag_p, cs_p)
            barrier()
            torch.cuda.synchronize()
            walls = []
            for _ in range(a.steps):
                t0 = time.perf_counter()
                re2 = eng.build_files(files, k, B, frag_p, cs_p)
                walls.append(time.perf_counter() - t0)
            ems = 1000.0 * sum(walls) / len(walls)
            ems = max_over_ranks(ems, world, "cuda")
            e2e = {"value": job_kmers / (ems / 1000.0), "unit": "k-mers/s", "ms_per_step": ems,
                   # phase 1 here spans the host inflate/parse it overlaps with;
                   # the rest of the call after phase 2 is the output copies and writes
                   "last_call_ms": {"phase1_with_read": re2.ms_phase1, "phase2": re2.ms_phase2,
                                    "outputs_after_phase2": re2.ms_outputs, "total": re2.ms_total},
                   "h2d_bytes_per_step": int(re2.h2d_bytes), "d2h_bytes_per_step": int(re2.d2h_bytes),
                   "path": "cdbg_gpu_build_files: %d gzip FASTA files (%.2f GB) -> frag_unitigs.bin (%.2f GB) + "
                           ".color_sets in %s, wall time per call" % (len(files), gz_bytes / 1e9,
                                                                       re2.frag_nbytes / 1e9, os.path.dirname(fdir))}
        finally:
            shutil.rmtree(fdir, ignore_errors=True)
        # the same build from pinned host sequences to host outputs
        step(host_batch, True)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            re3 = step(host_batch, True)
        e1.record(stream)
        torch.cuda.synchronize()
        hms = max_over_ranks(e0.elapsed_time(e1) / a.steps, world, "cuda")
        e2e_host = {"value": job_kmers / (hms / 1000.0), "unit": "k-mers/s", "ms_per_step": hms,
                    "h2d_bytes_per_step": int(re3.h2d_bytes), "d2h_bytes_per_step": int(re3.d2h_bytes),
                    "path": "cdbg_gpu_build: pinned host ASCII sequences -> host outputs"}

    # ---- plain path: one bucket per batch (one launch sequence per bucket)
    plain = None
    if a.compare_plain or skewed:
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        rp = step(dev_batch, False, batch_occ=1)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        plain = {"ms_per_step": pms, "value": kmers / (pms / 1000.0), "phase_ms": {"phase1": rp.ms_phase1,
                                                                                   "phase2": rp.ms_phase2},
                 "batched_over_plain": pms / ms}

    # ---- roofline: the dominant kernel with an algorithmic-bytes figure, and
    # the whole phase-1 + phase-2 path
    peak, peak_kind = peaks()
    w = 8 if k <= 31 else 16
    roof = None
    for name, (tot_ms, nl) in sorted(kstats.items(), key=lambda kv: -kv[1][0]):
        # bytes declared by the library's launch sites, else this file's per-unit figures
        alg = kbytes[name] / nl if kbytes.get(name) else algorithmic_bytes(name, r, w, a.steps, nl)
        if alg is None:
            continue
        per_launch_ms = tot_ms / nl
        ach = alg / (per_launch_ms / 1000.0) / 1e9
        tr = TRAFFIC_PER_UNIT.get(name) if k <= 31 else None  # captured with 64-bit k-mers
        ratio = TRAFFIC_RATIO.get(name)
        roof = {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak,
                "traffic": (tr[0] * units(name, r) * a.steps / nl) if tr else (alg * ratio[0] if ratio else None),
                "traffic_source": tr[1] if tr else (ratio[1] if ratio else None), "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": alg, "ms_per_launch": per_launch_ms,
                "launches_per_step": nl / a.steps, "share_of_step": tot_ms / (kms * a.steps),
                "timing": "CUDA events around each launch on its stream, over a second pass of the same "
                          "steps (%.1f ms per step with those events)" % kms}
        break
    path_bytes = path_algorithmic_bytes(r, w, rec_bytes)
    path_ach = path_bytes / (ms / 1000.0) / 1e9
    if roof is not None:
        roof["path"] = {"bytes_per_step": path_bytes, "achieved": path_ach, "frac": path_ach / peak,
                        "formula": "Nb/4 + 2*record_bytes + 2*Nocc*(w+4) + D*(w+8) + frag_bytes"}

    # ---- CPU baseline (reference, bounded sample), rank 0 at N = 1
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline and os.path.exists(REF_P12):
        R = ReferenceSample(a.workload, n_genomes, a.ref_slices, os.cpu_count() or 1, scale=a.genome_scale)
        try:
            km, s, det = R.run(0)
            cpu = {"value": km / s, "unit": "k-mers/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": R.describe(km), "step": det}
        finally:
            R.close()

    # ---- parity of the benchmarked path on the reference arm's sample: the
    # in-memory build from files against the reference's own process_buckets
    # (one thread: deterministic ids and order) on this build's bucket files
    check = None
    if rank == 0 and a.check:
        R = ReferenceSample(a.workload, n_genomes, a.ref_slices, os.cpu_count() or 1, scale=a.genome_scale)
        try:
            lst, skm = R.slice(0)
            sfiles = [l.strip() for l in open(lst) if l.strip()]
            wd = os.path.join(R.work, "check")
            bd = os.path.join(wd, "buckets")
            os.makedirs(bd)
            eng.phase1(sfiles, k, B, bd)
            r2 = os.path.join(ROOT, "oracle", "_ref", "ref_phase2" + ("-largek" if k > 31 else ""))
            t0 = time.time()
            rr = subprocess.run([r2, bd, str(B), str(k), str(n_genomes), "1", os.path.join(wd, "ref")],
                                capture_output=True, text=True)
            ref_s = time.time() - t0
            gf, gc = os.path.join(wd, "frag_unitigs.bin"), os.path.join(wd, "out.color_sets")
            eng.build_files(sfiles, k, B, gf, gc)
            same = lambda x, y: open(x, "rb").read() == open(y, "rb").read()
            check = {"sample": R.describe(skm).split(";")[0].replace("slice i mod", "slice 0 of"),
                     "kmers": skm, "ref_rc": rr.returncode, "ref_phase2_t1_s": ref_s,
                     "frag_unitigs_equal": rr.returncode == 0 and same(gf, os.path.join(wd, "ref", "frag_unitigs.bin")),
                     "color_sets_equal": rr.returncode == 0 and same(gc, os.path.join(wd, "ref", "out.color_sets")),
                     "frag_bytes": os.path.getsize(gf)}
        finally:
            R.close()

    if rank == 0:
        top = sorted(kstats.items(), key=lambda kv: -kv[1][0])[:20]
        line = {"metric": "phase1+2 k-mers/s", "value": value, "unit": "k-mers/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64" if k <= 31 else "u128", "data": "synthetic",
                "config": workload_config(a.workload, n_genomes, k, B, seq.nbytes, a.genome_scale),
                "parallelism": "replicas%d" % world,
                "workload_detail": {"kmers_per_step": int(job_kmers), "bases": int(seq.nbytes),
                                    "generate_s": gen_s, "tuning": eng.tuning()},
                "counts": {"supers": int(r.n_supers), "records": int(r.n_records), "occ": int(r.n_occ),
                           "distinct": int(r.n_distinct), "fragments": int(r.n_fragments),
                           "color_sets": int(r.n_color_sets), "frag_bytes": int(r.frag_nbytes)},
                "phase_ms": {"phase1": r.ms_phase1, "phase2": r.ms_phase2},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_host": e2e_host,
                "gpu_launches": int(launches),
                "autotune": tuned, "plain": plain, "check": check,
                "clocks": clocks,
                "kernels_ms_per_step": {kname: round(v[0] / a.steps, 3) for kname, v in top}}
        s = json.dumps(line)
        print(s)
        if a.out:
            with open(a.out, "w") as f:
                f.write(s + "\n")
    eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


# Algorithmic bytes per unit of each kernel (the unit is the count named in
# units()); probes, extra radix passes and re-reads are overhead, not counted.
def _per_unit(w):
    return {
        # 2-bit stream read once (1/4 B per base) + one cut entry written per
        # super-k-mer (minimizer value 8, run 4, position 4)
        "k_minimizers": None,  # two units, see algorithmic_bytes
        # one (k-mer, record) read per occurrence + one table entry per distinct k-mer
        "k_insert": None,
        "k_multi_pairs": ("occ", 4 + 4),          # occurrence slot read + pair written
        "k_ext_mask": ("distinct", w + 4 + 1),    # key + bucket read, mask written
        "k_links": ("distinct", w + 1 + 8 + 8),   # key + mask + recorded neighbours read, two links written
        "k_chain_paths": ("distinct", 8 + 1 + 1 + 4),  # links + flags + mask read, fragment element written
        "k_frag_write": ("frag_bytes", 1),        # fragment records written
    }


def units(name, r):
    u = {"occ": r.n_occ, "distinct": r.n_distinct, "frag_bytes": r.frag_nbytes,
         "supers": r.n_supers, "bases": r.n_bases}
    kind = {"k_minimizers": "bases", "k_insert": "occ"}.get(name)
    if kind is None:
        kind = _per_unit(8)[name][0]
    return u[kind]


def algorithmic_bytes(name, r, w, steps, launches):
    """Algorithmic bytes of one launch of `name` (per-unit figure x units)."""
    if name == "k_minimizers":
        v = r.n_bases / 4.0 + r.n_supers * 16
    elif name == "k_insert":
        v = r.n_occ * (w + 4) + r.n_distinct * (w + 8)
    else:
        pu = _per_unit(w).get(name)
        if pu is None:
            return None
        v = units(name, r) * pu[1]
    return v * steps / launches


def path_algorithmic_bytes(r, w, record_bytes):
    """Algorithmic bytes of one phase-1 + phase-2 pass: 2-bit input read, bucket
    records written and read back, one write + one read of every (k-mer,
    record) occurrence pair, one distinct k-mer table entry (key + cid + flags)
    and the fragment bytes written."""
    return (r.n_bases / 4.0 + 2 * record_bytes + 2 * r.n_occ * (w + 4) + r.n_distinct * (w + 8)
            + r.frag_nbytes)


# DRAM bytes per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum
# of one capture of the pangenome workload at 40 genomes, k=31, divided by the
# units that launch processed) and the summary under profiles/ it comes from.
# DRAM bytes per algorithmic byte of kernels whose launch sites declare their
# algorithmic bytes (one capture; the ratio carries to other sizes).
TRAFFIC_RATIO = {
    # first phase-1 pass at 40 genomes: 20,646,311 pairs, 495.5 MB algorithmic, 463.8 MB DRAM
    "k_rs_onesweep": (463810560 / 495511464, "profiles/phase12_top_kernels_pangenome40.md"),
}

TRAFFIC_PER_UNIT = {
    "k_minimizers": (1.691, "profiles/phase12_top_kernels_pangenome40.md"),   # per base
    "k_insert": (61.321, "profiles/phase12_top_kernels_pangenome40.md"),      # per occurrence
    "k_ext_mask": (55.196, "profiles/phase12_top_kernels_pangenome40.md"),    # per distinct k-mer
    "k_frag_write": (3.688, "profiles/phase12_top_kernels_pangenome40.md"),   # per fragment byte
}


# ---------------------------------------------------------------- serving
def serving_requests(n_req, seed=7, host_bytes=0):
    """The serving stream's requests: per request its own seeded ancestor, 2-300
    genomes (log-uniform) of 0.5-8 Mbp (log-uniform), 0.1-2% divergence, k in
    {31, 63}; returns ([(seq, off, colors, n_genomes, k, kmers)] in pinned
    host memory, number of distinct collections).  When the collections of
    all requests would not fit in `host_bytes` of host memory, the first ones
    that fit are generated and the later requests submit them again in turn
    (each submission is still a whole build)."""
    import numpy as np
    import torch
    from cdbg_gpu import synth
    rng = np.random.default_rng(seed)
    shapes = []
    for i in range(n_req):
        n = int(round(np.exp(rng.uniform(np.log(2), np.log(300)))))
        k = int(rng.choice([31, 63]))
        shapes.append((n, k))
    out, used = [], 0
    for i, (n, k) in enumerate(shapes):
        p, _, _, _ = synth.preset("serving", seed=10000 + i)
        seq, lens, per = synth.collection(p, n)
        if host_bytes and out and used + seq.nbytes > host_bytes:
            break
        used += seq.nbytes
        off = np.zeros(len(lens) + 1, dtype=np.uint64)
        off[1:] = np.cumsum(lens)
        colors = np.repeat(np.arange(n, dtype=np.uint32), per)
        out.append((torch.from_numpy(seq).pin_memory(), torch.from_numpy(off.view(np.int64)).pin_memory(),
                    torch.from_numpy(colors.view(np.int32)).pin_memory(), n, k, count_kmers(lens, k)))
    distinct = len(out)
    return [out[i % distinct] for i in range(n_req)], distinct


def serve_stream(reqs, arrivals, slots, budget, B, batch_occ):
    """Submit each request at its arrival time to a server; returns per-request
    (latency s, queue wait s, device ms) and the makespan."""
    from cdbg_gpu import native
    import queue
    import threading
    srv = native.Server(0, slots=slots, hbm_budget=budget)
    try:
        t0 = srv.stats()["clock_s"]
        ids = queue.Queue()
        res, errs = [], []

        # a waiter collects and releases each request as it finishes (in
        # submission order), so finished outputs do not pile up in host memory
        def waiter():
            while True:
                item = ids.get()
                if item is None:
                    return
                rid, arr = item
                try:
                    r = srv.wait(rid, outputs=False)
                except Exception as ex:  # keep draining: every request is released
                    errs.append(str(ex))
                    continue
                if r["status"] != 0:
                    errs.append("request failed: " + r["error"])
                res.append((r["t_done"] - arr, r["t_start"] - arr, r["ms_device"], r["t_done"]))

        wt = threading.Thread(target=waiter)
        wt.start()
        try:
            for (seq, off, col, n, k, _), at in zip(reqs, arrivals):
                while srv.stats()["clock_s"] - t0 < at:
                    time.sleep(0.0005)
                b = native.SeqBatch(seq.data_ptr(), seq.numel(), off.data_ptr(), col.data_ptr(), col.numel(), 0)
                ids.put((srv.submit(b, k, B, n, batch_occ=batch_occ), t0 + at))
        finally:
            ids.put(None)
            wt.join()
        if errs:
            raise RuntimeError(errs[0])
        st = srv.stats()
    finally:
        srv.close()
    makespan = max(x[3] for x in res) - (t0 + arrivals[0])
    return res, makespan, st


def main_serving(a):
    import numpy as np
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    t = time.time()
    try:
        import psutil
        host = int(psutil.virtual_memory().available * 0.3)
    except Exception:
        host = 64 << 30
    reqs, distinct = serving_requests(a.requests, host_bytes=host)
    gen_s = time.time() - t
    rng = np.random.default_rng(11)
    arrivals = np.cumsum(rng.exponential(1.0 / a.rate, size=len(reqs)))
    arrivals -= arrivals[0]
    budget = int(a.budget_gb * (1 << 30))
    B = a.serving_buckets
    kmers = sum(r[5] for r in reqs)
    slot_list = [int(x) for x in str(a.slots).split(",") if x]
    # warm-up: the whole stream once through a server (device memory pool and
    # pinned output buffers reach their steady-state sizes), not timed
    serve_stream(reqs, [0.0] * len(reqs), max(slot_list), budget, B, 0)

    def summary(res, makespan, st):
        lat = np.array([x[0] for x in res])
        km = sum(r[5] for r in reqs[:len(res)])
        return {"builds_per_s": len(res) / makespan, "kmers_per_s": km / makespan,
                "makespan_s": makespan, "latency_p50_s": float(np.percentile(lat, 50)),
                "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.percentile([x[1] for x in res], 50)),
                "peak_running": st["peak_running"], "peak_reserved_gb": st["peak_reserved_bytes"] / 2 ** 30}

    by_slots = {}
    for sl in slot_list:
        by_slots[sl] = summary(*serve_stream(reqs, arrivals, sl, budget, B, 0))
    best = max(by_slots, key=lambda sl: by_slots[sl]["builds_per_s"])
    serving = dict(by_slots[best], slots=best)
    # the plain path (one request at a time, one bucket per batch) is an order
    # of magnitude slower: it serves the stream's first requests only
    npl = min(len(reqs), a.plain_requests)
    plain = None if a.no_plain else summary(*serve_stream(reqs[:npl], list(arrivals[:npl]), 1, budget, B, 1))
    if plain:
        plain["requests"] = npl
    one_slot = by_slots.get(1)
    line = {"metric": "serving builds/s", "value": serving["builds_per_s"], "unit": "builds/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "serving: %d requests (Poisson %.1f/s), 2-300 genomes x 0.5-8 Mbp log-uniform, "
                                   "k in {31, 63}, %d buckets, slots %s, %.0f GB HBM budget"
                                   % (len(reqs), a.rate, B, a.slots, a.budget_gb),
                       "total_kmers": kmers, "generate_s": gen_s, "distinct_collections": distinct},
            "serving": serving, "by_slots": by_slots, "plain_sequential": plain,
            "speedup_vs_plain": (serving["builds_per_s"] / plain["builds_per_s"]) if plain else None,
            "speedup_vs_one_slot_batched": (serving["builds_per_s"] / one_slot["builds_per_s"]) if one_slot else None}
    print(json.dumps(line))
    if a.out:
        with open(a.out, "w") as f:
            f.write(json.dumps(line) + "\n")
    return 0


def main_seed(a):
    """Round 0 of the stitch (cdbg_gpu_stitch_seed) over the frag_unitigs.bin of
    the pangenome build: fragments/s, and the reference's own seed
    (oracle/_ref/ref_seed, all host cores) on the same file beside it.  Rank 0
    only (a per-GPU figure; the build's bench line carries the replicas)."""
    import numpy as np
    import torch
    from cdbg_gpu import native, synth
    rank, local, world = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    p, n_genomes, k, blog2 = synth.preset("pangenome", seed=1, scale=a.genome_scale)
    if a.genomes:
        n_genomes = a.genomes
    B = a.seed_buckets
    seq, lens, per = synth.collection(p, n_genomes)
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    colors = np.repeat(np.arange(n_genomes, dtype=np.uint32), per)
    eng = native.Engine(local)
    h_seq = torch.from_numpy(seq).pin_memory()
    h_off = torch.from_numpy(off.view(np.int64)).pin_memory()
    h_col = torch.from_numpy(colors.view(np.int32)).pin_memory()
    batch = native.SeqBatch(h_seq.data_ptr(), seq.nbytes, h_off.data_ptr(), h_col.data_ptr(), len(colors), 0)
    r = eng.build(batch, k, 1 << blog2, n_genomes)
    n_frag_bytes = r.frag_nbytes
    frags = torch.empty(n_frag_bytes + 16, dtype=torch.uint8).pin_memory()
    ctypes_memmove(frags.data_ptr(), r.frag_bytes, n_frag_bytes)
    del h_seq, h_off, h_col, seq
    eng.trim()
    base = scratch_base(4 * n_frag_bytes + (8 << 30)) or tempfile.gettempdir()
    work = tempfile.mkdtemp(prefix="cdbg_seed_", dir=base)
    try:
        calls = [0]

        def step():
            # each call writes a fresh directory, as a build's stitch does; the
            # files are removed after the call, outside its wall time
            d = os.path.join(work, "gpu%d" % calls[0])
            calls[0] += 1
            r = eng.stitch_seed((frags.data_ptr(), n_frag_bytes), k, d, num_buckets=B,
                                closed_path=os.path.join(d, "closed.bin"))
            shutil.rmtree(d, ignore_errors=True)
            return r

        for _ in range(max(a.warmup, 3)):
            st = step()
        clk = ClockSampler(local)
        clk.start()
        l0 = native.launch_count()
        runs = [step() for _ in range(a.steps)]
        launches = (native.launch_count() - l0) // max(1, a.steps)
        clocks = clk.stop()
        eng.profile(True)
        step()
        kstats = eng.kernel_stats()
        eng.profile(False)
        nf = runs[0]["fragments"]
        ms_dev = statistics.mean(x["ms_device"] for x in runs)
        ms_tot = statistics.mean(x["ms_total"] for x in runs)
        st = runs[-1]
        hbm, src = peaks()
        seed_k = {kk: v for kk, v in kstats.items() if kk.startswith("k_seed")}
        top = max(seed_k, key=lambda kk: seed_k[kk][0])
        # algorithmic bytes of one launch of the top kernel
        # (k_seed_info: every record byte read, its offset, 32 bytes of sizes,
        # bucket and state written; k_seed_write: every record byte read, the
        # tigs and closed unitigs written, 48 bytes of per-fragment offsets,
        # sizes and state read)
        if top == "k_seed_info":
            alg = n_frag_bytes + 8 * (nf + 1) + 32 * nf
        elif top == "k_seed_write":
            alg = n_frag_bytes + st["round0_bytes"] + st["closed_nbytes"] + 48 * nf
        else:
            alg = None
        top_ms = seed_k[top][0] / max(1, seed_k[top][1])
        achieved = alg / (top_ms * 1e6) if alg else None
        # the reference's seed on the same file, all host cores
        ref = None
        exe = os.path.join(ROOT, "oracle", "_ref", "ref_seed")
        if not a.no_cpu_baseline and os.path.exists(exe):
            fp = os.path.join(work, "frag_unitigs.bin")
            frags[:n_frag_bytes].numpy().tofile(fp)
            threads = os.cpu_count() or 1
            out = subprocess.run([exe, fp, str(k), str(B), str(threads), os.path.join(work, "ref")],
                                 capture_output=True, text=True, check=True).stdout
            sec = float(re.search(r"seconds=([0-9.]+)", out).group(1))
            ref = {"value": nf / sec, "unit": "fragments/s", "cores": threads, "kind": "reference",
                   "sample": "the whole frag file (%d fragments, %.2f GB), one run, %d round-store buckets"
                             % (nf, n_frag_bytes / 1e9, B), "seconds": sec}
        line = {"metric": "stitch round-0 seed fragments/s", "value": nf / (ms_dev / 1e3), "unit": "fragments/s",
                "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms_dev,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                "config": {"workload": "stitch seed: the frag_unitigs.bin of the pangenome build (%d genomes x "
                                       "~4.8 Mbp, k=%d), %d round-store buckets" % (n_genomes, k, B),
                           "fragments": nf, "frag_bytes": n_frag_bytes, "routed": st["routed"],
                           "closed_fragments": st["closed_fragments"], "closed_unitigs": st["closed_unitigs"],
                           "round0_bytes": st["round0_bytes"], "round0_file_bytes": st["round0_file_bytes"],
                           "l2": "inputs larger than L2 (%.1f GB of fragments)" % (n_frag_bytes / 1e9)},
                "e2e": {"value": nf / (ms_tot / 1e3), "unit": "fragments/s", "ms_per_call": ms_tot,
                        "ms_scan": statistics.mean(x["ms_scan"] for x in runs),
                        "ms_device": ms_dev, "ms_files": statistics.mean(x["ms_files"] for x in runs),
                        "h2d_bytes_per_step": n_frag_bytes, "d2h_bytes_per_step": st["round0_bytes"]
                        + st["closed_nbytes"], "what": "host frag bytes in, round-0 files and closed-unitig file "
                        "written (%s)" % ("tmpfs" if base == "/dev/shm" else "disk")},
                "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm if achieved else None, "traffic": None,
                             "peak_source": src, "ms_per_launch": top_ms},
                "kernels_ms": {kk: v[0] for kk, v in seed_k.items()},
                "cpu_baseline": ref, "gpu_launches": launches, "clocks": clocks}
        print(json.dumps(line))
        if a.out:
            with open(a.out, "w") as f:
                f.write(json.dumps(line) + "\n")
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return 0


def ctypes_memmove(dst, src, n):
    import ctypes
    ctypes.memmove(dst, src, n)


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        sys.exit(reference_arm(args))
    if args.workload == "serving":
        sys.exit(main_serving(args))
    if args.workload == "stitch-seed":
        sys.exit(main_seed(args))
    sys.exit(main_gpu(args))
