"""Builds libmgk.so (the CUDA kernels + C ABI) and the mgkde_tiled host driver
in-tree, for sm_100a only.

  python -m mgpukde_tiled_b200.build [--verbose-ptxas]

Outputs go to mgpukde_tiled_b200/_lib/.  nvcc cross-compiles here without a
GPU; the built files travel with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "_lib")
OBJ = os.path.join(PKG, "_build")
CU_SOURCES = ["api.cu", "index.cu", "density.cu", "boundary.cu", "edge.cu", "loo.cu", "serve.cu", "stream.cu", "tune.cu", "adaptive.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(out: str, deps) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(REPO, "include", "mgk.h"))
    common = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "-I", os.path.join(REPO, "include")]
    if verbose_ptxas:
        common += ["-Xptxas", "-v"]

    def compile_one(src):
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        if not force and not verbose_ptxas and _newer(o, [s, *headers]):
            return o, ""
        p = subprocess.run(common + ["-c", s, "-o", o], capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{p.stdout}\n{p.stderr}")
        return o, p.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, CU_SOURCES))
    if verbose_ptxas:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    so = os.path.join(LIB, "libmgk.so")
    if force or not _newer(so, objs):
        subprocess.run([nvcc(), *ARCH, "-shared", "-o", so, *objs, "-lcudart", "-lpthread"], check=True)
    cli_src = os.path.join(CSRC, "cli.cpp")
    cli = os.path.join(LIB, "mgkde_tiled")
    if os.path.exists(cli_src) and (force or not _newer(cli, [cli_src, so, *headers])):
        cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(REPO, "include"),
                        "-I", CSRC, "-I", os.path.join(cuda, "include"), cli_src, "-o", cli, "-L", LIB, "-lmgk",
                        "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN"],
                       check=True)
    return so


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.force))
