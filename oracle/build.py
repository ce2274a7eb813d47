"""Builds the C++ oracle (oracle/_build/libvipe_oracle.so) with g++ — test infrastructure."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libvipe_oracle.so"


def build(verbose: bool = False) -> Path:
    srcs = [HERE / "ba_oracle.cpp"]  # the ref_*_shim.cpp files belong to build_ref.py
    if LIB.exists() and all(s.stat().st_mtime < LIB.stat().st_mtime for s in srcs):
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-O2", "-pthread", "-fPIC", "-std=c++17", "-shared", "-o", str(LIB), *map(str, srcs)]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
