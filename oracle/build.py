"""Builds the oracle's C++ restatement (oracle/_build/liboracle.so) and, when the
reference tree is present, the reference-code drivers (oracle/_ref/, via
oracle/ref/Makefile). Test infrastructure only."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"
# The reference tree the drivers compile from: RAYON_REFERENCE, by default the
# read-only checkout at /root/reference.
REFERENCE = Path(os.environ.get("RAYON_REFERENCE", "/root/reference"))


def build_oracle(verbose: bool = False) -> Path:
    src = HERE / "rb_oracle.cpp"
    deps = [src, HERE.parent / "rayon_b200" / "csrc" / "rb_rng.h", HERE.parent / "include" / "rayon_b200_scene.h"]
    if OUT.exists() and OUT.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-ffp-contract=off", "-o", str(OUT) + ".tmp",
           str(src)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(str(OUT) + ".tmp", OUT)
    return OUT


def build_reference(verbose: bool = False) -> bool:
    """Compile the reference drivers into oracle/_ref/ (only where the reference tree exists)."""
    if not (REFERENCE / "src" / "rayon").is_dir():
        return False
    r = subprocess.run(["make", "-C", str(HERE / "ref"), f"REF={REFERENCE}"], capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout[-2000:] + r.stderr[-4000:])
    return r.returncode == 0


if __name__ == "__main__":
    print(build_oracle(verbose=True))
    print("reference drivers:", build_reference(verbose=True))
