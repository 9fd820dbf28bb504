"""Build the native library of the B200 render path.

Compiles rayon_b200/csrc/*.cu for sm_100a with nvcc and *.cpp with g++, then
links rayon_b200/_lib/librayon_b200.so (CUDA runtime linked statically).
Incremental: an object is rebuilt when its source or any header in csrc/ is
newer. No torch extension machinery and no JIT cache: the .so lives in-tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
CSRC = ROOT / "csrc"
BUILD = ROOT / "_build"
LIBDIR = ROOT / "_lib"
LIB = LIBDIR / "librayon_b200.so"
INCLUDE = ROOT.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Intersection arithmetic is compiled with the same fast-math flags as the
# reference CUDA renderer (CMakeLists.txt:196-209) so hit decisions match.
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--use_fast_math", "-Xcompiler", "-fPIC",
    "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread", f"-I{INCLUDE}", f"-I{CSRC}"]


def _newest_header() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... ({r.returncode})")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    hdr = _newest_header()
    jobs = []
    objs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr):
            continue
        if src.suffix == ".cu":
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++", *CXX_FLAGS, "-I/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
        jobs.append(cmd)
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(lambda c: _run(c, verbose or ptxas_info), jobs))
    if jobs or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              "-Xcompiler", "-pthread"], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
