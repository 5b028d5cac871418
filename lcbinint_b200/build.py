"""Builds the in-tree CUDA library lcbinint_b200/liblcbinint_b200.so for sm_100a.

    python -m lcbinint_b200.build [--force] [-v]

Every .cu file under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``.  Files are compiled
with ``--fmad=false`` (no multiply-add contraction) so the FP64 paths
reproduce the reference's IEEE arithmetic bit for bit; files whose name ends
in ``_fast.cu`` opt into contraction (the FP32 ray paths, whose error is
reported against the FP64 result instead).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "liblcbinint_b200.so"
OBJ = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _flags(src: Path) -> list[str]:
    fmad = "--fmad=true" if src.stem.endswith("_fast") else "--fmad=false"
    return ARCH + ["-lineinfo", "-O3", fmad, "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                   "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}", "-Xptxas", "-warn-spills"]


def _deps(src: Path) -> list[Path]:
    return [src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    cc = nvcc()
    jobs = []
    for src in srcs:
        obj = OBJ / (src.stem + ".o")
        if force or _stale(obj, _deps(src)):
            jobs.append([cc, "-c", str(src), "-o", str(obj)] + _flags(src))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
        for cmd, r in zip(jobs, results):
            if verbose or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {cmd[2]}")
    objs = [OBJ / (s.stem + ".o") for s in srcs]
    if force or jobs or _stale(LIB, objs):
        link = [cc, "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH + ["-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(" ".join(link) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.v))
