"""CPU: the build server's admission gate (host/admission.hpp), compiled
into a small driver: budget reservations, arrival order, the slot limit and
the always-admit-one rule of the reference's bucket-process gate
(phase2_bucket_process/bucket_walker.hpp:631-671)."""
import os
import shutil
import subprocess

import pytest

from conftest import PKG

DRIVER = r'''
#include <cstdio>
#include "admission.hpp"
using cdbg::serve::admission_gate;
static void show(admission_gate& g) {
    uint64_t id, grant;
    while (g.admit(id, grant)) std::printf("start %llu %llu\n", (unsigned long long)id, (unsigned long long)grant);
    std::printf("state %llu %u %zu\n", (unsigned long long)g.reserved(), g.running(), g.waiting());
}
int main() {
    admission_gate g(100, 3);
    g.arrive(1, 40); g.arrive(2, 40); g.arrive(3, 40); g.arrive(4, 150); g.arrive(5, 10);
    show(g);          // 1, 2 start; 3 does not fit (80 + 40 > 100)
    g.finish(40);     // 1 done
    show(g);          // 3 starts; 4 (150 > budget) waits for an empty GPU
    g.finish(40); g.finish(40);
    show(g);          // 4 runs alone with the whole budget
    g.finish(100);
    show(g);          // 5 starts
    admission_gate s(1000, 2);
    s.arrive(1, 1); s.arrive(2, 1); s.arrive(3, 1);
    show(s);          // the slot limit: two run
    cdbg::serve::memory_model m;
    std::printf("need %llu\n", (unsigned long long)m.need(1000));
}
'''

EXPECT = """start 1 40
start 2 40
state 80 2 3
start 3 40
state 80 2 2
start 4 100
state 100 1 1
start 5 10
state 10 1 0
start 1 1
start 2 1
state 2 2 1
need %d
""" % (24 * 1000 + (2 << 30))


def test_admission_gate(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    src = tmp_path / "gate.cpp"
    src.write_text(DRIVER)
    exe = str(tmp_path / "gate")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(PKG, "host"), str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    assert out == EXPECT
