"""Build ``ksim_b200/lib/libksim_b200.so`` in-tree with nvcc for sm_100a.

Run ``python -m ksim_b200.build`` (``-v`` prints ptxas register / spill
reports).  The library links the CUDA runtime statically, so it only needs the
driver at run time; it travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "libksim_b200.so"
BUILD = PKG / "lib" / "_obj"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["kernels.cu", "api.cu", "peak.cu", "batch.cu", "serve.cu", "noalloc.cu", "noise.cu", "image.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: Path, obj: Path, verbose: bool) -> str:
    if src.suffix == ".cu":
        cmd = [nvcc(), "-c", str(src), "-o", str(obj), *ARCH, "-O3", "-std=c++17", "-lineinfo",
               "-fmad=false", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I", str(CSRC)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-c", str(src), "-o", str(obj), "-O3", "-std=c++17", "-fPIC",
               "-ffp-contract=off", "-I", str(CSRC), "-I", "/usr/local/cuda/include"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "ksim_b200.h"]
    newest_dep = max(p.stat().st_mtime for p in deps)
    jobs = []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, newest_dep):
            jobs.append((s, o))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for (s, _), log in zip(jobs, ex.map(lambda so: _compile(so[0], so[1], verbose), jobs)):
            if verbose and log.strip():
                print(f"== {s.name}\n{log}", file=sys.stderr)
    objs = [str(BUILD / (s.name + ".o")) for s in srcs]
    if jobs or not LIB.exists():
        cmd = [nvcc(), "-shared", "-o", str(LIB), *objs, *ARCH, "-Xcompiler", "-fPIC", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-f", "--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))


if __name__ == "__main__":
    main()
