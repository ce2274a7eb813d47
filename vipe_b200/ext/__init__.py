"""Drop-in replacements for the reference's ``vipe.ext`` extension modules.

    from vipe_b200.ext import slam_ext, droid_net_ext, lietorch_ext, corr_ext

mirror ``from vipe.ext import slam_ext, droid_net_ext, lietorch_ext, corr_ext``
(vipe/ext/__init__.py:39-45 of the reference).  ``install_as_vipe_ext()``
registers them under ``vipe.ext`` in ``sys.modules`` so unchanged reference
code (GraphBuffer, FactorGraph, the lietorch groups, the AOT tracker's
spatial correlation sampler) imports them.
"""

from __future__ import annotations

import importlib
import sys
import types

__all__ = ["slam_ext", "droid_net_ext", "lietorch_ext", "corr_ext", "install_as_vipe_ext"]

_MODULES = ("slam_ext", "droid_net_ext", "lietorch_ext", "corr_ext")


def __getattr__(name):
    if name in _MODULES:
        mod = importlib.import_module(f"{__name__}.{name}")
        globals()[name] = mod
        return mod
    raise AttributeError(name)


def install_as_vipe_ext() -> types.ModuleType:
    """Registers this package's modules as ``vipe.ext.{slam_ext,droid_net_ext,lietorch_ext,corr_ext}``."""
    vipe = sys.modules.get("vipe") or types.ModuleType("vipe")
    vipe.__path__ = getattr(vipe, "__path__", [])
    ext = sys.modules.get("vipe.ext") or types.ModuleType("vipe.ext")
    ext.__path__ = getattr(ext, "__path__", [])
    for name in _MODULES:
        mod = importlib.import_module(f"{__name__}.{name}")
        setattr(ext, name, mod)
        sys.modules[f"vipe.ext.{name}"] = mod
    vipe.ext = ext
    sys.modules["vipe"] = vipe
    sys.modules["vipe.ext"] = ext
    return ext
