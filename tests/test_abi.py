"""The C-ABI library loads on a machine without a GPU and exports every entry
point that include/vipe_b200.h declares (no compute calls are made here)."""

import re
from pathlib import Path

from vipe_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "vipe_b200.h"


def _declared() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vipe_\w+)\s*\(", text, flags=re.M))


def test_header_declares_the_bound_signatures():
    declared = _declared()
    assert len(declared) >= 39
    assert declared == set(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in _declared() if getattr(lib, n, None) is None]
    assert not missing, missing
    assert _lib.missing_symbols() == []


def test_status_strings():
    assert _lib.status_string(0)
    assert "index" in _lib.status_string(_lib.VIPE_ERR_INDEX).lower()


def test_argument_checks_run_before_any_device_work():
    """Entry points reject bad sizes and pointers with a status before touching the GPU, so
    these calls are safe without one (null device pointers are never dereferenced)."""
    import ctypes

    lib = _lib.load()
    null = ctypes.c_void_p(0)
    # write probe: null destination, size not a multiple of 16
    assert lib.vipe_hbm_write_probe(null, 16, null) == _lib.VIPE_ERR_ARG
    assert lib.vipe_hbm_write_probe(ctypes.c_void_p(16), 15, null) == _lib.VIPE_ERR_ARG
    # coordinate gradient of the volume lookup: negative sizes
    assert lib.vipe_corr_index_coords_backward(0, null, null, null, -1, 4, 4, 4, 4, 3, null, null) == \
        _lib.VIPE_ERR_ARG
    # indexed lookup backward: no levels, too many channels, missing outputs
    h2 = (ctypes.c_int * 1)(8)
    w2 = (ctypes.c_int * 1)(8)
    lv = (ctypes.c_void_p * 1)(16)
    args = dict(dtype=0, f1=ctypes.c_void_p(16), lv=lv, h2=h2, w2=w2, L=1, B=1, Nf=2, M=1, H=8, W=8, C=32, r=3)

    def call(**kw):
        a = {**args, **kw}
        g1 = kw.get("g1", ctypes.c_void_p(16))
        gl = kw.get("gl", lv)
        return lib.vipe_altcorr_index_backward(a["dtype"], a["f1"], a["lv"], a["h2"], a["w2"], a["L"], null, null,
                                               null, null, a["B"], a["Nf"], a["M"], a["H"], a["W"], a["C"], a["r"],
                                               0, g1, gl, null, null)

    assert call(L=0) == _lib.VIPE_ERR_ARG
    assert call(C=512) == _lib.VIPE_ERR_CAPACITY
    assert call(r=4) == _lib.VIPE_ERR_CAPACITY
    assert call(g1=null) == _lib.VIPE_ERR_ARG


def test_pyramid_and_window_checks_without_a_gpu():
    """The feature-pyramid entry points reject level counts, channel counts and types before any
    device work; the BA workspace query accepts windows of up to 1024 poses and refuses more."""
    import ctypes

    lib = _lib.load()
    null = ctypes.c_void_p(0)
    outs = (ctypes.c_void_p * 5)(16, 16, 16, 16, 16)
    assert lib.vipe_corr_pyramid_nhwc(_lib.VIPE_F16, null, 1, 128, 48, 64, 5, outs, null) == _lib.VIPE_ERR_ARG
    assert lib.vipe_corr_pyramid_nhwc(_lib.VIPE_F16, null, 1, 12, 48, 64, 4, outs, null) == _lib.VIPE_ERR_ARG
    assert lib.vipe_corr_pyramid_nhwc(_lib.VIPE_F64, null, 1, 128, 48, 64, 4, outs, null) == _lib.VIPE_ERR_DTYPE
    assert lib.vipe_corr_pyramid_nhwc(_lib.VIPE_F16, null, 1, 128, 4, 64, 4, outs, null) == _lib.VIPE_ERR_ARG
    assert lib.vipe_corr_pyramid_nhwc_backward(_lib.VIPE_F32, null, 1, 128, 48, 64, 0, null, null) == \
        _lib.VIPE_ERR_ARG
    assert lib.vipe_slam_ba_workspace_size(1025, 8, 8, 3000, 1024, 1, 1025) > 0
    assert lib.vipe_slam_ba_workspace_size(1026, 8, 8, 3000, 1025, 1, 1026) == 0


def test_install_as_vipe_ext_registers_every_reference_module():
    """`from vipe.ext import slam_ext, droid_net_ext, lietorch_ext, corr_ext` resolves to this
    package's modules, with the reference's bound function names (slam.cpp:41-55,
    droid.cpp:75-81, lietorch.cpp:306-336, correlation_sampler.cpp:82-85)."""
    import sys

    saved = {k: sys.modules.get(k) for k in list(sys.modules) if k == "vipe" or k.startswith("vipe.")}
    try:
        from vipe_b200.ext import install_as_vipe_ext

        install_as_vipe_ext()
        from vipe.ext import corr_ext, droid_net_ext, lietorch_ext, slam_ext  # noqa: F401

        for name in ("ba", "ba_extended", "frame_distance", "projmap", "depth_filter", "iproj"):
            assert callable(getattr(slam_ext, name))
        for name in ("altcorr_forward", "altcorr_backward", "altcorr_index_forward", "corr_index_forward",
                     "corr_index_backward"):
            assert callable(getattr(droid_net_ext, name))
        for name in ("expm", "logm", "inv", "mul", "adj", "adjT", "act", "act4", "as_matrix", "projector", "Jinv"):
            assert callable(getattr(lietorch_ext, name))
        assert callable(corr_ext.forward) and callable(corr_ext.backward)
    finally:
        for k in [k for k in sys.modules if k == "vipe" or k.startswith("vipe.")]:
            del sys.modules[k]
        sys.modules.update({k: v for k, v in saved.items() if v is not None})


def test_proximity_edge_checks_without_a_gpu():
    import ctypes

    lib = _lib.load()
    null = ctypes.c_void_p(0)
    assert lib.vipe_slam_proximity_edges_workspace_size(5, 6, 10) == 0  # t0 < t1
    assert lib.vipe_slam_proximity_edges_capacity(0, 0, 10, 2, 48, 0) == 50
    # more than 1.7 M candidates: refused before any device work
    rc = lib.vipe_slam_proximity_edges(ctypes.c_void_p(16), null, null, 0, 0, 0, 1400, 2, 3, ctypes.c_float(22.0),
                                       16 * 1400, 0, ctypes.c_void_p(16), ctypes.c_void_p(16), 1 << 20,
                                       ctypes.c_void_p(16), ctypes.c_void_p(16), 1 << 30, null)
    assert rc == _lib.VIPE_ERR_CAPACITY


def test_fused_correlation_entry_checks_without_a_gpu():
    import ctypes

    lib = _lib.load()
    null = ctypes.c_void_p(0)
    lv = (ctypes.c_void_p * 4)(16, 16, 16, 16)
    one = ctypes.c_void_p(16)
    # three levels, a 64-bit type: refused before any device work
    assert lib.vipe_corr_encoder_lookup(_lib.VIPE_F16, lv, 3, one, 1, 48, 64, one, null, one, one, null) == \
        _lib.VIPE_ERR_ARG
    assert lib.vipe_corr_encoder_lookup(_lib.VIPE_F64, lv, 4, one, 1, 48, 64, one, null, one, one, null) == \
        _lib.VIPE_ERR_DTYPE
    # volume adjoint: more than 128 channels, H*W not a multiple of 128
    assert lib.vipe_corr_volume_backward(_lib.VIPE_F16, _lib.VIPE_F16, one, one, lv, 1, 256, 48, 64, 4, one, one,
                                         one, null) == _lib.VIPE_ERR_ARG
    assert lib.vipe_corr_volume_backward(_lib.VIPE_F16, _lib.VIPE_F16, one, one, lv, 1, 128, 10, 10, 1, one, one,
                                         one, null) == _lib.VIPE_ERR_ARG
