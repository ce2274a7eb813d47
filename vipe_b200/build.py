"""Builds the vipe_b200 CUDA library (sm_100a only) in-tree.

    python -m vipe_b200.build          # -> vipe_b200/_lib/libvipe_b200.so

The library is plain CUDA C++ with an extern "C" ABI (include/vipe_b200.h);
it links the CUDA runtime statically and has no torch dependency, so the
shared object loads into any process (torch, ctypes, cgo, ...).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libvipe_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=default",
    "--expt-relaxed-constexpr",
    "-DVIPE_BUILD",
]


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]
    for c in cand:
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found; the vipe_b200 CUDA library cannot be built")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _needs_build(objs: list[tuple[Path, Path]]) -> bool:
    if not LIB.exists():
        return True
    lib_t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(p.stat().st_mtime > lib_t for p in deps)


def build(verbose: bool = False, force: bool = False, jobs: int | None = None) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    srcs = sources()
    objs = [(s, obj_dir / (s.stem + ".o")) for s in srcs]
    if not force and not _needs_build(objs):
        return LIB
    exe = nvcc()
    header_t = max(p.stat().st_mtime for p in list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))
    procs = []
    for src, obj in objs:
        if not force and obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, header_t):
            continue
        cmd = [exe, *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        if jobs and len([p for p in procs if p[1].poll() is None]) >= jobs:
            procs[0][1].wait()
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        msg = "\n".join(f"--- {s.name}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [exe, *ARCH, "-shared", "-o", str(tmp), *[str(o) for _, o in objs], "-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(verbose=True, force=force))
