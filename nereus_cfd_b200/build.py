"""Builds the B200 library in-tree: nereus_cfd_b200/libnereus_b200.so, sm_100a only.

    python -m nereus_cfd_b200.build [--verbose]

nb_exact.cu, nb_relabel.cu and nb_bc.cu are compiled with -fmad=false (their results must round like the reference's host
code); the solver kernels keep fused multiply-adds. The object files go to nereus_cfd_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnereus_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                 "-I" + os.path.join(os.path.dirname(HERE), "include")]
SOURCES = {
    "nb_exact.cu": ["-fmad=false"],
    "nb_kernels.cu": [],
    "nb_tail.cu": [],
    "nb_pairs.cu": [],
    "nb_split.cu": [],
    "nb_solver.cu": [],
    "nb_capi.cu": [],
    "nb_noalloc.cu": [],
    "nb_relabel.cu": ["-fmad=false"],
    "nb_bc.cu": ["-fmad=false"],
    "nb_server.cu": [],
    "nb_batch.cu": [],
}
HEADERS = ["nb_device.cuh", "nb_batch.cuh", "nb_kernels.h", "nb_solver.h", "nb_guard.h"]


def _newest_input() -> float:
    paths = [os.path.join(CSRC, s) for s in list(SOURCES) + HEADERS]
    paths.append(os.path.join(os.path.dirname(HERE), "include", "nereus_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


def up_to_date() -> bool:
    return os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input()


def _compile(src: str, extra, verbose: bool) -> str:
    obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
    cmd = [NVCC] + COMMON + extra + (["-Xptxas", "-v"] if verbose else []) + ["-c", os.path.join(CSRC, src),
                                                                               "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), SOURCES.items()))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
