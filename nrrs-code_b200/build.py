"""Build libnrrs_b200.so (sm_100a) in-tree with nvcc.

Usage: python nrrs-code_b200/build.py [--force]

Objects go to nrrs-code_b200/_build/, the library to nrrs-code_b200/lib/. Both are git-ignored
and travel with the source tree. Only files whose sources (or the shared headers) changed are
recompiled.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "lib" / "libnrrs_b200.so"
INCLUDE = HERE.parent / "include"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "nrrs.h"])


def _compile(src: Path, extra: list[str]) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = list(extra or [])
    if verbose:
        extra += ["-Xptxas", "-v"]
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    hdr_mtime = max(p.stat().st_mtime for p in headers())
    todo = []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        if force or verbose or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime):
            todo.append(src)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for obj, log in ex.map(lambda s: _compile(s, extra), todo):
            if verbose and log:
                sys.stderr.write(f"== {obj.name}\n{log}")
    objs = [BUILD / (s.name + ".o") for s in sources()]
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", *map(str, objs), "-o", str(LIB),
               "-lcudart", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="pass -Xptxas -v")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))
