"""CPU: the C++ adapter the repository's integration guide prints (its first
C++ block) compiles against the reference's headers and this project's
header, and links against libcdbg_gpu.so (no GPU needed to link)."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

REF = os.environ.get("CDBG_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
LIB = os.path.join(ROOT, "cdbg-builder_b200", "libcdbg_gpu.so")

USE = r'''
#include "gpu_phases.hpp"
int main(int argc, char**) {
    if (argc < 99) return 0;  // link check only
    cdbg::gpu::engine g(0);
    std::vector<std::string> files;
    std::vector<uint64_t> unc;
    cdbg::gpu::ingest_bucketed(g, files, 31, 0, 1024, "tmp", 1, &unc);
    cdbg::streaming_color_set_dict d(4, "x.color_sets");
    cdbg::gpu::process_buckets(g, "tmp", 1024, 31, 4, "tmp/frag_unitigs.bin", d, false, 1);
    cdbg::gpu::build_in_memory(g, files, 31, 0, 1024, "tmp/frag_unitigs.bin", "x.color_sets", 1);
    std::atomic<uint64_t> done{0};
    cdbg::frag_unitig_writer sink("tmp/unitigs.bin");
    cdbg::gpu::stitch_from_frag_file(g, "tmp/frag_unitigs.bin", 31, "tmp", std::ref(sink), 1024, &done, 1);
}
'''


def test_adapter_compiles_and_links(tmp_path):
    if not os.path.isdir(os.path.join(REF, "include")):
        pytest.skip("reference sources not present")
    if not os.path.exists(LIB) or shutil.which("g++") is None:
        pytest.skip("library or g++ missing")
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    adapter = re.findall(r"```cpp\n(.*?)```", doc, re.S)[0]
    (tmp_path / "gpu_phases.hpp").write_text(adapter)
    (tmp_path / "use.cpp").write_text(USE)
    r = subprocess.run(["g++", "-std=c++17", "-O0", "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(REF, "include"), "-I" + os.path.join(ROOT, "oracle", "shim"),
                        "-I" + os.path.join(REF, "external"), str(tmp_path / "use.cpp"),
                        "-L" + os.path.dirname(LIB), "-lcdbg_gpu", "-l:liblz4.so.1", "-lz", "-pthread",
                        "-o", str(tmp_path / "use")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
