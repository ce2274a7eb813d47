"""Builds the reference's own correlation extensions from their unchanged sources.

TEST INFRASTRUCTURE ONLY: the modules built here are the checker that the GPU
parity tests run beside vipe_b200 on the same inputs; nothing in the product
imports them.

    python -m oracle.build_ref        # -> oracle/_ref/ref_droid_net_ext*.so, ref_corr_ext*.so

Sources, read where they lie in the reference checkout (never copied):
  * ref_droid_net_ext: csrc/droid_net_ext/{altcorr_kernel.cu, correlation_kernels.cu,
    droid.cpp}, registered through `pybind_droid_net_ext` (droid.cpp:75-81);
  * ref_corr_ext: csrc/corr_ext/{correlation.cpp, correlation_sampler.cpp,
    correlation_cuda_kernel.cu}, registered through `pybind_corr_ext`.
Both need only ATen/torch (no Eigen), so they compile here; the reference's
slam_ext and lietorch_ext need Eigen 3.4, which the reference downloads at build
time (vipe/ext/specs.py:23), and cannot be built.  The compiler flags are the
reference's own (vipe/ext/specs.py: -O3 -DWITH_CUDA, --use_fast_math for CUDA)
plus the sm_100a target.  Each module gets a one-function pybind shim
(oracle/ref_*_shim.cpp) because the reference registers every extension into one
combined module (csrc/bind.cpp).

The built .so files live in oracle/_ref/ (git-ignored, shipped with the tree to
the GPU box, where the reference checkout does not exist); `load(name)` imports
a prebuilt module from there and never compiles.
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF = Path(os.environ.get("VIPE_REFERENCE_ROOT", "/root/reference"))

MODULES = {
    "ref_droid_net_ext": (
        ["csrc/droid_net_ext/altcorr_kernel.cu", "csrc/droid_net_ext/correlation_kernels.cu",
         "csrc/droid_net_ext/droid.cpp"],
        "ref_droid_net_shim.cpp",
    ),
    "ref_corr_ext": (
        ["csrc/corr_ext/correlation.cpp", "csrc/corr_ext/correlation_sampler.cpp",
         "csrc/corr_ext/correlation_cuda_kernel.cu"],
        "ref_corr_shim.cpp",
    ),
}

CFLAGS = ["-O3", "-DWITH_CUDA"]
CUDA_FLAGS = ["-O3", "-DWITH_CUDA", "--use_fast_math", "-gencode", "arch=compute_100a,code=sm_100a"]


def _built(name: str) -> Path | None:
    hits = sorted(OUT.glob(f"{name}*.so"))
    return hits[0] if hits else None


def build(verbose: bool = False, force: bool = False) -> list[Path]:
    """Compiles every module whose reference sources are present; returns the .so paths."""
    out = []
    for name, (srcs, shim) in MODULES.items():
        paths = [REF / s for s in srcs]
        have = _built(name)
        if not all(p.exists() for p in paths):
            if have is not None:
                out.append(have)
            continue
        newest = max(p.stat().st_mtime for p in paths + [HERE / shim, Path(__file__)])
        if have is not None and not force and have.stat().st_mtime > newest:
            out.append(have)
            continue
        from torch.utils import cpp_extension

        bdir = OUT / f"_build_{name}"
        bdir.mkdir(parents=True, exist_ok=True)
        # no GPU here: name the architecture instead of letting torch probe for one
        os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
        cpp_extension.load(
            name=name,
            sources=[str(p) for p in paths] + [str(HERE / shim)],
            extra_cflags=CFLAGS,
            extra_cuda_cflags=CUDA_FLAGS,
            build_directory=str(bdir),
            verbose=verbose,
            is_python_module=True,
        )
        so = bdir / f"{name}.so"
        dst = OUT / f"{name}.so"
        os.replace(so, dst)
        out.append(dst)
    return out


def load(name: str):
    """Imports the prebuilt reference module `name` from oracle/_ref (no compilation)."""
    if name in sys.modules:
        return sys.modules[name]
    so = _built(name)
    if so is None:
        raise ImportError(f"{name} is not built: run `python -m oracle.build_ref` where the reference checkout exists")
    import torch  # noqa: F401  (the module links against libtorch)

    loader = importlib.machinery.ExtensionFileLoader(name, str(so))
    spec = importlib.util.spec_from_file_location(name, str(so), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    sys.modules[name] = mod
    return mod


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv, force="--force" in sys.argv):
        print(p)
