"""Build libcpstep.so in-tree with nvcc for sm_100a.

Usage: python -m openatom_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcpstep.so")
BUILD = os.path.join(HERE, "_build")

import glob
from concurrent.futures import ThreadPoolExecutor

SOURCES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(CSRC, "*.cu"))) + [
    "layout.cpp", "statefile.cpp"]
HEADERS = sorted(os.path.basename(p) for p in glob.glob(os.path.join(CSRC, "*.cuh")))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fvisibility=hidden"]


def _deps():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(HERE, "..", "include", "cpstep.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(HERE, "..", "include"), "-c",
                                       os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        jobs.append((cmd, obj))

    def run(job):
        cmd, obj = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    objs = [obj for _, obj in jobs]
    nproc = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(nproc) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError("nvcc failed: " + cmd[-3])
    cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart", "-lz"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
