"""Build the native libraries in-tree.

* ``libcdbg_gpu.so``   CUDA kernels for sm_100a + host I/O + the C-ABI of
                       include/cdbg_gpu.h (nvcc, cudart linked statically).
* ``libcdbg_synth.so`` synthetic workload generator (g++).
* ``oracle/liboracle.so`` and, when the reference sources are present,
  ``oracle/_ref/*`` (the reference built from its own sources) -- test
  infrastructure, built here so the checker travels with the tree.

Run as ``python cdbg-builder_b200/build.py`` or through __graft_entry__.build().
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(NVCC))), "include")
CU_SOURCES = ["phase1.cu", "phase2.cu", "inflate.cu", "seed.cu", "capi.cu"]
HOST_SOURCES = ["io.cpp", "server.cpp", "shards.cpp"]
# the reference checkout sits beside this repository unless the variable says otherwise
REFERENCE = os.environ.get("CDBG_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _deps():
    out = []
    for d in (CSRC, HOST, INC):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".hpp", ".h")):
                out.append(os.path.join(d, f))
    return out


def build_gpu(force=False):
    lib = os.path.join(PKG, "libcdbg_gpu.so")
    deps = _deps()
    if not force and not _stale(lib, deps):
        return lib
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    for s in CU_SOURCES:
        o = os.path.join(OBJ, s + ".o")
        jobs.append([NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
                     "-I" + INC, "-c", os.path.join(CSRC, s), "-o", o])
    for s in HOST_SOURCES:
        o = os.path.join(OBJ, s + ".o")
        jobs.append(["g++", "-std=c++17", "-O3", "-fPIC", "-I" + INC, "-I" + CUDA_INC, "-c",
                     os.path.join(HOST, s), "-o", o])
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        list(ex.map(_run, jobs))
    objs = [j[-1] for j in jobs]
    tmp = lib + ".tmp"
    _run([NVCC, "-shared", *ARCH, "-o", tmp, *objs, "-lz", "-l:liblz4.so.1", "-lpthread"])
    os.replace(tmp, lib)
    return lib


def build_synth(force=False):
    lib = os.path.join(PKG, "libcdbg_synth.so")
    src = os.path.join(HOST, "synth.cpp")
    if force or _stale(lib, [src, os.path.join(INC, "cdbg_synth.h")]):
        _run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I" + INC, "-o", lib + ".tmp", src,
              "-lz", "-lpthread"])
        os.replace(lib + ".tmp", lib)
    return lib


def build_oracle(force=False):
    odir = os.path.join(ROOT, "oracle")
    lib = os.path.join(odir, "liboracle.so")
    src = os.path.join(odir, "oracle.cpp")
    if force or _stale(lib, [src]):
        _run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-o", lib + ".tmp", src, "-lz",
              "-l:liblz4.so.1"])
        os.replace(lib + ".tmp", lib)
    if os.path.isdir(os.path.join(REFERENCE, "include")):
        _run(["make", "-s", "-j8", "ref", "REF=" + REFERENCE], cwd=odir)
    return lib


def build_all(force=False):
    with ThreadPoolExecutor(max_workers=3) as ex:
        futs = [ex.submit(build_gpu, force), ex.submit(build_synth, force), ex.submit(build_oracle, force)]
        return [f.result() for f in futs]


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
