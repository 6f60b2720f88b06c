"""Builds libdmap_b200.so in place: every CUDA source for sm_100a with nvcc.

The translation units with FP64 arithmetic that must round like the
reference (pyramid.cu, setup.cu, walk64.cu, walk32_exact.cu for the paths
that run the FP64 leaf, shade.cu, tess.cu, emitter.cu)
are compiled with -fmad=false so that each double operation rounds on its
own, as the reference's CPU build does; FP32 code there asks for fused
multiply-adds explicitly (fmaf, __fmaf_ru). walk32.cu (the FP32 walk
rounds) is compiled with contraction.
Usage: python -m dmap_b200.build [-j N] [--force]
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
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libdmap_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC)]
EXACT_FP64 = {"pyramid.cu", "setup.cu", "walk64.cu", "walk32_exact.cu", "shade.cu", "tess.cu", "emitter.cu"}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _compile(src: Path, extra) -> Path:
    obj = BUILD / (src.stem + ".o")
    flags = ARCH + COMMON + (["-fmad=false"] if src.name in EXACT_FP64 else []) + list(extra)
    cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + flags
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [ROOT / "include" / "dmap_b200.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, jobs: int = 0, extra=()) -> Path:
    if not force and not _stale():
        return LIB
    BUILD.mkdir(exist_ok=True)
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-o", str(tmp)] + [str(o) for o in objs] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    print(build(a.force or a.ptxas_verbose, a.j, extra))


if __name__ == "__main__":
    main()
