"""CPU: `bench.py --impl reference` (the reference's own phase 1 + phase 2,
timed on bounded samples of the benchmark's own collection) prints one JSON
line with the bench contract's keys, on the same metric and workload config
as the GPU arm."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT, ref_bin


def test_reference_arm_prints_one_contract_line():
    if not ref_bin("ref_phase12", 31):
        pytest.skip("oracle/_ref not built")
    # a 6-genome collection, two steps over slices 1/4 of every genome
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--genomes", "6", "--ref-slices", "4"], capture_output=True, text=True,
                       cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "phase1+2 k-mers/s" and d["unit"] == "k-mers/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    # the label names what ran: the 6-genome collection, sampled as stated
    assert d["config"]["workload"].startswith("pangenome: 6 genomes")
    assert d["config"]["genomes"] == 6 and d["config"]["k"] == 31 and d["config"]["buckets"] == 4096
    assert "1/4 of every one of the 6 genomes" in d["sample"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "k-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
