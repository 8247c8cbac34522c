"""Build libcalypso_b200.so in-tree with nvcc for sm_100a.

Usage: python -m calypso_b200.build   (or calypso_b200.build.build())
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcalypso_b200.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["cb2_api.cu", "cb2_tables.cu", "cb2_rj.cu", "cb2_legendre_f64.cu",
           "cb2_fft.cu", "cb2_legendre_mixed.cu", "cb2_static_scratch.cu",
           "cb2_tune.cu", "cb2_closure.cu", "cb2_cn.cu", "cb2_boundary.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "calypso_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, jobs: int = 6) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    procs, objs = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, s.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, src):
            cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            if len(procs) >= jobs:
                _wait(procs)
                procs = []
    _wait(procs)
    need_link = not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)
    if need_link:
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", "/usr/bin/g++",
               "-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lcudart", "-lgomp"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
    return LIB


def _wait(procs):
    errs = []
    for name, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append(f"{name}:\n{out.decode(errors='replace')}")
        elif out and b"warning" in out:
            sys.stderr.write(out.decode(errors="replace"))
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(verbose=True))
