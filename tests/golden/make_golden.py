"""Regenerate the golden fixtures in this directory from the reference itself.

The reference (jermp/cdbg-builder) is built from its own sources by
oracle/Makefile into oracle/_ref/.  This script writes small seeded FASTA
inputs, runs the reference's phase-1 harness (ref_phase1: its
ingest_file_bucketed / emit_super_kmers), the full reference binary with
--keep-tmp (its bucket files), and its phase-2 harness (ref_phase2: its
process_buckets + frag_unitig_writer + streaming_color_set_dict), and keeps
their outputs as fixtures:

  <case>/in/g*.fa(.fq)     inputs (filenames.txt lists them, relative)
  <case>/supers.bin        every super-k-mer occurrence (ref_phase1 dump)
  <case>/buckets.pack      the reference's bucket files (cdbg-build -t 1 --keep-tmp),
                           packed as [u64 size][file bytes] per bucket 0..B-1
  <case>/frag_unitigs.bin  ref_phase2 over those bucket files, 1 thread
  <case>/out.color_sets    finalized color sets of the same run
  <case>/meta.json         k, m, num_buckets, num_colors, counts
  <case>/seed_b64.pack     the reference's stitch round-0 files (ref_seed: its
                           ext_seed_round0_raw_par, 1 thread, 64 round-store
                           buckets) over frag_unitigs.bin, packed as
                           [u64 size][file bytes] per bucket 0..63 (size 0: no file)
  <case>/seed_closed.bin   the closed unitigs the same seed passed to its sink

Usage: python tests/golden/make_golden.py [--seed-only]   (needs oracle/_ref built;
--seed-only remakes the two seed fixtures from the existing frag_unitigs.bin)
"""
import json
import os
import shutil
import struct
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cdbg-builder_b200"))
from cdbg_gpu import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

CASES = {
    # name: (k, buckets_log2, genomes, synth overrides, seed, fastq)
    "tiny_k31": (31, 10, 3, dict(len_min=4000, len_max=4000, div_min=0.01, div_max=0.02, indels=3,
                                mobile_pool=2, mobile_min=300, mobile_max=600, contigs_min=1,
                                contigs_max=3, lowercase_runs=1, n_runs=1), 11, False),
    "tiny_k63": (63, 10, 3, dict(len_min=5000, len_max=5000, div_min=0.005, div_max=0.01, indels=3,
                                mobile_pool=2, mobile_min=300, mobile_max=600, repeat_pool=2,
                                repeats_per_genome=2, tandem_frac=0.02, contigs_min=1,
                                contigs_max=2), 12, False),
    "tiny_skew_fq": (31, 10, 4, dict(len_min=2000, len_max=6000, div_min=0.002, div_max=0.02,
                                    indels=2, lowcomp_frac=0.10, contigs_min=1, contigs_max=4,
                                    contigs_log=1, n_runs=1), 13, True),
}


def to_fastq(path_in, path_out):
    name, seq = None, []
    with open(path_in) as f, open(path_out, "w") as o:
        def flush():
            if name is not None:
                s = "".join(seq)
                o.write("@%s\n%s\n+\n%s\n" % (name, s, "I" * len(s)))
        for line in f:
            line = line.rstrip("\n")
            if line.startswith(">"):
                flush()
                name, seq = line[1:], []
            else:
                seq.append(line)
        flush()


def run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit("failed: %s\n%s\n%s" % (cmd, r.stdout, r.stderr))
    return r.stdout


def make_case(name, spec):
    k, bl, n, over, seed, fastq = spec
    d = os.path.join(HERE, name)
    shutil.rmtree(d, ignore_errors=True)
    os.makedirs(os.path.join(d, "in"))
    p = synth.make_params(seed=seed, **over)
    synth.write_fasta(p, n, os.path.join(d, "in"))
    names = ["g%d.fa" % i for i in range(n)]
    if fastq:
        for i, nm in enumerate(names):
            src = os.path.join(d, "in", nm)
            to_fastq(src, os.path.join(d, "in", "g%d.fq" % i))
            os.remove(src)
        names = ["g%d.fq" % i for i in range(n)]
    with open(os.path.join(d, "in", "filenames.txt"), "w") as f:
        f.write("".join(nm + "\n" for nm in names))
    big = k > 31
    abslist = os.path.join(d, "abs_filenames.txt")
    with open(abslist, "w") as f:
        f.write("".join(os.path.join(d, "in", nm) + "\n" for nm in names))
    B = 1 << bl
    m = 12 if k == 31 else 14
    run([os.path.join(REF, "ref_phase1" + ("-largek" if big else "")), abslist, str(k), "0", str(B),
         os.path.join(d, "supers.bin")])
    tmp = os.path.join(d, "_tmp")
    out = run([os.path.join(REF, "cdbg-build" + ("-largek" if big else "")), "-i", abslist, "-k", str(k),
               "-o", os.path.join(tmp, "out"), "-t", "1", "-b", str(bl), "-d", os.path.join(tmp, "w"),
               "--keep-tmp"])
    with open(os.path.join(d, "buckets.pack"), "wb") as pk:
        for b in range(B):
            data = open(os.path.join(tmp, "w", "bucket_%d.bin" % b), "rb").read()
            pk.write(struct.pack("<Q", len(data)) + data)
    meta_txt = open(os.path.join(tmp, "out.metadata.txt")).read()
    r2 = run([os.path.join(REF, "ref_phase2" + ("-largek" if big else "")), os.path.join(tmp, "w"),
              str(B), str(k), str(n), "1", os.path.join(tmp, "p2")])
    shutil.copy(os.path.join(tmp, "p2", "frag_unitigs.bin"), d)
    shutil.copy(os.path.join(tmp, "p2", "out.color_sets"), d)
    shutil.copy(os.path.join(tmp, "out.fa"), os.path.join(d, "final.fa"))
    stats = dict(kv.split("=") for kv in r2.split() if "=" in kv and kv.strip("=") == kv)
    meta = dict(k=k, m=m, num_buckets=B, num_colors=n,
                metadata=dict(l.split("=") for l in meta_txt.split()),
                phase2={kk: v for kk, v in stats.items() if kk != "seconds"})
    with open(os.path.join(d, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    shutil.rmtree(tmp)
    os.remove(abslist)


SEED_BUCKETS = 64


def make_seed(name, k):
    d = os.path.join(HERE, name)
    tmp = os.path.join(d, "_seed")
    shutil.rmtree(tmp, ignore_errors=True)
    run([os.path.join(REF, "ref_seed" + ("-largek" if k > 31 else "")), os.path.join(d, "frag_unitigs.bin"),
         str(k), str(SEED_BUCKETS), "1", tmp])
    with open(os.path.join(d, "seed_b%d.pack" % SEED_BUCKETS), "wb") as pk:
        for b in range(SEED_BUCKETS):
            f = os.path.join(tmp, "stitch_r0_b%d.bin" % b)
            data = open(f, "rb").read() if os.path.exists(f) else b""
            pk.write(struct.pack("<Q", len(data)) + data)
    shutil.copy(os.path.join(tmp, "closed.bin"), os.path.join(d, "seed_closed.bin"))
    shutil.rmtree(tmp)


def unpack_seed(case_dir):
    """{bucket: round-0 file bytes} of a case's seed fixture."""
    data = open(os.path.join(case_dir, "seed_b%d.pack" % SEED_BUCKETS), "rb").read()
    out, p = {}, 0
    for b in range(SEED_BUCKETS):
        (n,) = struct.unpack_from("<Q", data, p)
        p += 8
        if n:
            out[b] = data[p:p + n]
        p += n
    return out


if __name__ == "__main__":
    for name, spec in CASES.items():
        if "--seed-only" not in sys.argv:
            make_case(name, spec)
        make_seed(name, spec[0])
        print("wrote", name)


def unpack_buckets(case_dir, out_dir):
    """Write the packed reference bucket files of a case into out_dir."""
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(case_dir, "buckets.pack"), "rb") as f:
        data = f.read()
    p = 0
    b = 0
    while p < len(data):
        (n,) = struct.unpack_from("<Q", data, p)
        p += 8
        with open(os.path.join(out_dir, "bucket_%d.bin" % b), "wb") as o:
            o.write(data[p:p + n])
        p += n
        b += 1
    return b
