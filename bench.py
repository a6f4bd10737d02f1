"""Benchmark: phase 1 + phase 2 k-mers/s on one B200 (or N replicas).

Workload (default): the pangenome configuration -- 1000 synthetic genomes of
~4.8 Mbp derived from one seeded ancestor (0.1-2% SNPs, 20 indels, one mobile
insert, 1-200 contigs), k = 31, m = 12, 4096 buckets.  A step is one full pass
of phase 1 + phase 2 over the whole collection (all k-mers), producing the
frag spill and the color classes.

  value   k-mers/s with the sequences already resident in HBM and the outputs
          left on the device (cdbg_gpu_build, on_device = 1).
  e2e     the same call with pinned host input buffers and host outputs: the
          H2D copy of the sequences and the D2H copy of the frag bytes and the
          color-set words are inside every timed step.

Time is measured with CUDA events on the stream the library launches on
(the engine runs on a torch stream), max over ranks.  `--impl reference`
times the reference's own CPU build (oracle/_ref/cdbg-build, built from its
sources) on a bounded sample with all host cores.  With --gpus N each rank
builds its own collection (independent replicas, weak scaling).
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
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "cdbg-build")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="pangenome")
    ap.add_argument("--genomes", type=int, default=0, help="override genome count (0 = workload's)")
    ap.add_argument("--cpu-sample-genomes", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch-occ", type=int, default=0)
    ap.add_argument("--table-slots-q", type=int, default=0,
                    help="k-mer table slots per 4 occurrences, 5..16 (0 = library default)")
    ap.add_argument("--autotune", action="store_true",
                    help="run the autotuner on the workload before timing (default for skewed)")
    ap.add_argument("--compare-plain", action="store_true",
                    help="also time one step of the plain one-bucket-per-batch path (default for skewed)")
    ap.add_argument("--out", default="")
    # serving workload
    ap.add_argument("--requests", type=int, default=48, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=30.0, help="serving: Poisson arrivals per second")
    ap.add_argument("--slots", default="1,2,3,4",
                    help="serving: concurrent builds; a list is swept and the best is reported")
    ap.add_argument("--no-plain", action="store_true", help="serving: skip the plain one-at-a-time run")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: HBM budget")
    ap.add_argument("--serving-buckets", type=int, default=1024)
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
def run_reference_sample(genomes, k, blog2, threads, seed, workdir):
    """One reference build of `genomes` genomes; returns (kmers, seconds p1+p2, detail)."""
    from cdbg_gpu import synth
    p, _, _, _ = synth.preset("pangenome", seed=seed)
    ind = os.path.join(workdir, "in")
    if not os.path.exists(os.path.join(ind, "filenames.txt")):
        synth.write_fasta(p, genomes, ind, gzip_level=1)
    _, lens, _ = synth.collection(p, genomes)
    kmers = count_kmers(lens, k)
    out = os.path.join(workdir, "o")
    shutil.rmtree(out, ignore_errors=True)
    os.makedirs(out)
    r = subprocess.run([REF_BIN, "-i", os.path.join(ind, "filenames.txt"), "-k", str(k), "-o",
                        os.path.join(out, "out"), "-t", str(threads), "-b", str(blog2), "-d",
                        os.path.join(out, "tmp")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed: " + r.stderr[-500:])
    t1 = float(re.search(r"\[bucket-write\] ([0-9.eE+-]+) s", r.stdout).group(1))
    t2 = float(re.search(r"\[bucket-process\] ([0-9.eE+-]+) s", r.stdout).group(1))
    return kmers, t1 + t2, {"bucket_write_s": t1, "bucket_process_s": t2}


def workload_name(n_genomes, k, B, workload="pangenome"):
    from cdbg_gpu.native import best_m
    shape = {
        "pangenome": "%d genomes x 4.8 Mbp (0.1-2%% SNPs, 1-200 contigs)",
        "small": "%d genomes x 5.0 Mbp (0.5%% SNPs, 20 indels, 1-3 contigs)",
        "largek": "%d genomes x 4.8 Mbp + 2%% tandem repeats + 200 shared 1-5 kbp repeats each",
        "skewed": "%d genomes x 1-6 Mbp log-uniform, 10%% homopolymer/dinucleotide runs",
    }.get(workload, "%d genomes")
    return "%s: %s, k=%d, m=%d, %d buckets" % (workload, shape % n_genomes, k, best_m(k), B)


def reference_arm(a):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cdbg-build not built"}))
        return 0
    threads = os.cpu_count() or 1
    k, blog2 = 31, 12
    g = a.cpu_sample_genomes
    work = tempfile.mkdtemp(prefix="cdbg_ref_")
    try:
        for _ in range(a.warmup):
            run_reference_sample(g, k, blog2, threads, 1, work)
        vals, secs = [], []
        kmers = 0
        for _ in range(a.steps):
            kmers, s, det = run_reference_sample(g, k, blog2, threads, 1, work)
            vals.append(kmers / s)
            secs.append(s)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    v = statistics.median(vals)
    sample = "%d of 1000 pangenome genomes (~4.8 Mbp, gzip FASTA), %d k-mers per step" % (g, kmers)
    line = {"impl": "reference", "metric": "phase1+2 k-mers/s", "value": v, "unit": "k-mers/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000 * statistics.median(secs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": workload_name(1000, k, 1 << blog2), "sample": sample,
                       "parallelism": "reference cdbg-build -t %d" % threads},
            "cpu_baseline": {"value": v, "unit": "k-mers/s", "cores": threads, "kind": "reference",
                             "sample": sample},
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

    p, n_genomes, k, blog2 = synth.preset(a.workload, seed=1 + rank)
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
    if a.table_slots_q:
        eng.set_tuning(table_slots_q=a.table_slots_q)
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

    # ---- e2e: pinned host buffers in, host outputs out
    e2e = None
    if not a.no_e2e:
        step(host_batch, True)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            re2 = step(host_batch, True)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / a.steps
        ems = max_over_ranks(ems, world, "cuda")
        e2e = {"value": job_kmers / (ems / 1000.0), "unit": "k-mers/s", "ms_per_step": ems,
               "h2d_bytes_per_step": int(re2.h2d_bytes), "d2h_bytes_per_step": int(re2.d2h_bytes)}

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
    if rank == 0 and world == 1 and not a.no_cpu_baseline and os.path.exists(REF_BIN):
        work = tempfile.mkdtemp(prefix="cdbg_cpu_")
        try:
            km, s, det = run_reference_sample(a.cpu_sample_genomes, k, blog2, os.cpu_count() or 1, 1, work)
            cpu = {"value": km / s, "unit": "k-mers/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "%d of %d genomes, %d k-mers, reference cdbg-build -t %d -b %d (%s)" % (
                       a.cpu_sample_genomes, n_genomes, km, os.cpu_count(), blog2, json.dumps(det))}
        finally:
            shutil.rmtree(work, ignore_errors=True)

    if rank == 0:
        top = sorted(kstats.items(), key=lambda kv: -kv[1][0])[:20]
        line = {"metric": "phase1+2 k-mers/s", "value": value, "unit": "k-mers/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64" if k <= 31 else "u128", "data": "synthetic",
                "config": {"workload": workload_name(n_genomes, k, B, a.workload),
                           "kmers_per_step": int(job_kmers), "bases": int(seq.nbytes),
                           "l2": "inputs (%.1f GB) larger than L2" % (seq.nbytes / 1e9),
                           "parallelism": "replicas%d" % world, "generate_s": gen_s,
                           "tuning": eng.tuning()},
                "counts": {"supers": int(r.n_supers), "records": int(r.n_records), "occ": int(r.n_occ),
                           "distinct": int(r.n_distinct), "fragments": int(r.n_fragments),
                           "color_sets": int(r.n_color_sets), "frag_bytes": int(r.frag_nbytes)},
                "phase_ms": {"phase1": r.ms_phase1, "phase2": r.ms_phase2},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "autotune": tuned, "plain": plain,
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
        "k_links": ("distinct", w + 4 + 1 + 8),   # key + bucket + mask read, two links written
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
    # first phase-1 pass at 40 genomes: 20,646,311 pairs, 495.5 MB algorithmic, 472.2 MB DRAM
    "k_rs_downsweep": (472166144 / 495511464, "profiles/phase12_top_kernels_pangenome40.md"),
}

TRAFFIC_PER_UNIT = {
    "k_minimizers": (1.691, "profiles/phase12_top_kernels_pangenome40.md"),   # per base
    "k_insert": (61.321, "profiles/phase12_top_kernels_pangenome40.md"),      # per occurrence
    "k_ext_mask": (55.196, "profiles/phase12_top_kernels_pangenome40.md"),    # per distinct k-mer
    "k_frag_write": (3.688, "profiles/phase12_top_kernels_pangenome40.md"),   # per fragment byte
}


# ---------------------------------------------------------------- serving
def serving_requests(n_req, seed=7):
    """The serving stream's requests: per request its own seeded ancestor, 2-300
    genomes (log-uniform) of 0.5-8 Mbp (log-uniform), 0.1-2% divergence, k in
    {31, 63}; returns [(seq, off, colors, n_genomes, k)] in pinned host memory."""
    import numpy as np
    import torch
    from cdbg_gpu import synth
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_req):
        n = int(round(np.exp(rng.uniform(np.log(2), np.log(300)))))
        k = int(rng.choice([31, 63]))
        p, _, _, _ = synth.preset("serving", seed=10000 + i)
        seq, lens, per = synth.collection(p, n)
        off = np.zeros(len(lens) + 1, dtype=np.uint64)
        off[1:] = np.cumsum(lens)
        colors = np.repeat(np.arange(n, dtype=np.uint32), per)
        out.append((torch.from_numpy(seq).pin_memory(), torch.from_numpy(off.view(np.int64)).pin_memory(),
                    torch.from_numpy(colors.view(np.int32)).pin_memory(), n, k, count_kmers(lens, k)))
    return out


def serve_stream(reqs, arrivals, slots, budget, B, batch_occ):
    """Submit each request at its arrival time to a server; returns per-request
    (latency s, queue wait s, device ms) and the makespan."""
    from cdbg_gpu import native
    srv = native.Server(0, slots=slots, hbm_budget=budget)
    try:
        t0 = srv.stats()["clock_s"]
        ids = []
        for (seq, off, col, n, k, _), at in zip(reqs, arrivals):
            while srv.stats()["clock_s"] - t0 < at:
                time.sleep(0.0005)
            b = native.SeqBatch(seq.data_ptr(), seq.numel(), off.data_ptr(), col.data_ptr(), col.numel(), 0)
            ids.append((srv.submit(b, k, B, n, batch_occ=batch_occ), t0 + at))
        res = []
        for rid, arr in ids:
            r = srv.wait(rid, outputs=False)
            if r["status"] != 0:
                raise RuntimeError("request failed: " + r["error"])
            res.append((r["t_done"] - arr, r["t_start"] - arr, r["ms_device"], r["t_done"]))
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
    reqs = serving_requests(a.requests)
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
        return {"builds_per_s": len(res) / makespan, "kmers_per_s": kmers / makespan,
                "makespan_s": makespan, "latency_p50_s": float(np.percentile(lat, 50)),
                "latency_p99_s": float(np.percentile(lat, 99)),
                "queue_wait_p50_s": float(np.percentile([x[1] for x in res], 50)),
                "peak_running": st["peak_running"], "peak_reserved_gb": st["peak_reserved_bytes"] / 2 ** 30}

    by_slots = {}
    for sl in slot_list:
        by_slots[sl] = summary(*serve_stream(reqs, arrivals, sl, budget, B, 0))
    best = max(by_slots, key=lambda sl: by_slots[sl]["builds_per_s"])
    serving = dict(by_slots[best], slots=best)
    plain = None if a.no_plain else summary(*serve_stream(reqs, arrivals, 1, budget, B, 1))
    line = {"metric": "serving builds/s", "value": serving["builds_per_s"], "unit": "builds/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "serving: %d requests (Poisson %.1f/s), 2-300 genomes x 0.5-8 Mbp log-uniform, "
                                   "k in {31, 63}, %d buckets, slots %s, %.0f GB HBM budget"
                                   % (len(reqs), a.rate, B, a.slots, a.budget_gb),
                       "total_kmers": kmers, "generate_s": gen_s},
            "serving": serving, "by_slots": by_slots, "plain_sequential": plain,
            "speedup_vs_plain": (serving["builds_per_s"] / plain["builds_per_s"]) if plain else None}
    print(json.dumps(line))
    if a.out:
        with open(a.out, "w") as f:
            f.write(json.dumps(line) + "\n")
    return 0


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        sys.exit(reference_arm(args))
    if args.workload == "serving":
        sys.exit(main_serving(args))
    sys.exit(main_gpu(args))
