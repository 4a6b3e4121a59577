"""Build libspx.so (sm_100a) in-tree.

    python fenicsx-micromagnetics_b200/build.py [--force] [-v]

Every translation unit under csrc/ is compiled by nvcc for sm_100a and linked
into spinfemx_b200/libspx.so, next to the Python package that loads it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "_build"
LIB = HERE / "spinfemx_b200" / "libspx.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers():
    return sorted(list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h")))


def _compile(src: Path, verbose: bool, extra):
    obj = OUT_DIR / (src.name + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, *FLAGS, "-x", "cu", *ARCH, *extra, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, extra=None) -> Path:
    extra = list(extra or [])
    OUT_DIR.mkdir(exist_ok=True)
    srcs = sources()
    newest_dep = max(p.stat().st_mtime for p in srcs + headers() + [Path(__file__)])
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest_dep:
        return LIB
    todo = []
    for s in srcs:
        obj = OUT_DIR / (s.name + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(s.stat().st_mtime, max(
                h.stat().st_mtime for h in headers())) or extra:
            todo.append(s)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, verbose, extra), todo))
    objs = [str(OUT_DIR / (s.name + ".o")) for s in srcs]
    cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    ap.add_argument("-D", action="append", default=[], help="extra preprocessor definition (tuning builds)")
    a = ap.parse_args()
    ex = ["-Xptxas", "-v"] if a.ptxas_v else []
    ex += [f"-D{d}" for d in a.D]
    print(build(force=a.force or a.ptxas_v or bool(a.D), verbose=a.v or a.ptxas_v, extra=ex))
    sys.exit(0)
