"""Build libturbch_b200.so (sm_100a) in-tree.

    python -m turbchannel_b200.build        # or turbchannel_b200.build.build()

Every .cu under csrc/ is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` in parallel, then
linked into turbchannel_b200/libturbch_b200.so next to this file.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libturbch_b200.so")
DRIVER_SRC = os.path.join(HERE, "driver", "turbch_run.cpp")
DRIVER = os.path.join(HERE, "turbch_run")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]


def _newer(dst: str, srcs: list[str]) -> bool:
    if not os.path.exists(dst):
        return False
    t = os.path.getmtime(dst)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(HERE, "..", "include", "turbch.h"), os.path.join(HERE, "..", "include", "turbch_les.h")]
    objs = []
    cmds = []
    for s in sources:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if not _newer(o, [s] + headers):
            cmds.append([NVCC, *ARCH, *FLAGS, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(run, cmds))
    if cmds or not _newer(LIB, objs):
        run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    # the command-line driver links the library with an rpath to its directory
    if not _newer(DRIVER, [DRIVER_SRC, LIB] + headers):
        run(["g++", "-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), DRIVER_SRC, "-o", DRIVER,
             "-L", HERE, "-lturbch_b200", f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
