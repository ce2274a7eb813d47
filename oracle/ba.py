"""Python front of the BA oracle (oracle/ba_oracle.cpp) — TEST INFRASTRUCTURE ONLY.

The C++ restates the reference's fused BA (vipe csrc/slam_ext/geom_kernels.cu
:1626-1847) in FP32 (use_fp64=False, the reference's own arithmetic) or in
all-FP64 (the accuracy oracle).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import build

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        D = ctypes.POINTER(ctypes.c_double)
        L = ctypes.POINTER(ctypes.c_int64)
        I = ctypes.c_int
        F = ctypes.c_double
        _lib.oracle_ba.restype = I
        _lib.oracle_ba.argtypes = [I, D, D, D, D, D, D, D, L, L, D, I, I, I, I, I, I, I, I, F, F, I, F, I, F, F, F, I,
                                   D, D, D]
        _lib.oracle_ba_index.restype = I
        _lib.oracle_ba_index.argtypes = [L, L, I, I, I, L, L]
        _lib.oracle_schur_pairs.restype = ctypes.c_long
        _lib.oracle_schur_pairs.argtypes = [L, L, I, I, I, L, L, L]
        _lib.oracle_set_threads.restype = None
        _lib.oracle_set_threads.argtypes = [I]
        _lib.oracle_set_threads(1)
        _lib.oracle_set_camera.restype = None
        _lib.oracle_set_camera.argtypes = [I, ctypes.c_double]
        _lib.oracle_set_robust.restype = None
        _lib.oracle_set_robust.argtypes = [I, ctypes.c_double, D, I]
        _lib.oracle_accum_csr.restype = I
        _lib.oracle_accum_csr.argtypes = [L, L, I, I, I, L, L]
        _lib.oracle_set_backsub_all_rows.restype = None
        _lib.oracle_set_backsub_all_rows.argtypes = [I]
    return _lib


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def ba(p, *, fp64: bool, motion_only=False, optimize_intrinsics=False, intrinsics_lm=1e-6, intrinsics_ep=1e-6,
       intrinsics_scale=1.0, compute_energy=False, iterations=None, lm=None, ep=None, alpha=None,
       backsub_all_rows=False, robust_kind=0, robust_threshold=1.0, mu_schedule=None, camera_model=0,
       distortion=0.0):
    """Runs the oracle on a workloads.BAProblem-like object (CPU tensors or arrays).

    backsub_all_rows=True keeps the depth back-substitution rows of pose t0, which the
    reference's fused kernel skips (geom_kernels.cu:1186) and its generic solver keeps.
    robust_kind 1/2/3 (Huber, Tukey, GNC-TLS with mu_schedule[i] for iteration i) multiplies
    each flow channel's weight by the generic solver's kernel of its residual
    (vipe/slam/ba/kernel.py:40-153, terms.py:73-75).  camera_model 1 projects through the MEI
    camera with k1 = distortion (vipe/utils/cameras.py:220-330).
    Returns dict(poses, disps, intrinsics, dx, dz, energy) as float64 arrays.
    """
    poses = _d(np.asarray(p.poses, dtype=np.float64)).copy()
    disps = _d(np.asarray(p.disps, dtype=np.float64)).copy()
    intr = _d(np.asarray(p.intrinsics, dtype=np.float64)).copy()
    sens = _d(np.asarray(p.disps_sens, dtype=np.float64))
    tg = _d(np.asarray(p.targets, dtype=np.float64))
    wt = _d(np.asarray(p.weights, dtype=np.float64))
    eta = _d(np.asarray(p.eta, dtype=np.float64))
    ii = np.ascontiguousarray(np.asarray(p.ii), dtype=np.int64)
    jj = np.ascontiguousarray(np.asarray(p.jj), dtype=np.int64)
    act = _d(np.asarray(p.depth_active, dtype=np.float64))
    N, H, W = disps.shape
    E = ii.shape[0]
    K = eta.shape[0]
    iters = p.iterations if iterations is None else iterations
    P = p.t1 - p.t0
    dx = np.zeros((P, 6))
    dz = np.zeros((K, H * W))
    en = np.zeros(max(iters, 1))
    D = ctypes.c_double
    L = ctypes.c_int64
    lib().oracle_set_backsub_all_rows(int(bool(backsub_all_rows)))
    mu = np.ascontiguousarray(np.asarray([] if mu_schedule is None else mu_schedule, dtype=np.float64))
    lib().oracle_set_robust(int(robust_kind), float(robust_threshold), _p(mu, D) if mu.size else None, int(mu.size))
    lib().oracle_set_camera(int(camera_model), float(distortion))
    rc = lib().oracle_ba(
        1 if fp64 else 0, _p(poses, D), _p(disps, D), _p(intr, D), _p(sens, D), _p(tg, D), _p(wt, D), _p(eta, D),
        _p(ii, L), _p(jj, L), _p(act, D), N, H, W, E, K, p.t0, p.t1, iters,
        p.lm if lm is None else lm, p.ep if ep is None else ep, int(motion_only),
        p.alpha if alpha is None else alpha, int(optimize_intrinsics), intrinsics_lm, intrinsics_ep,
        intrinsics_scale, int(compute_energy), _p(dx, D), _p(dz, D), _p(en, D),
    )
    lib().oracle_set_backsub_all_rows(0)
    lib().oracle_set_robust(0, 1.0, None, 0)
    lib().oracle_set_camera(0, 0.0)
    if rc != 0:
        raise RuntimeError(f"oracle_ba failed with code {rc}")
    return dict(poses=poses, disps=disps, intrinsics=intr, dx=dx, dz=None if motion_only else dz,
                energy=en[:iters] if compute_energy else np.zeros(0))


def index(ii, jj, t0, t1):
    """(kx, kk_exp) of the reference's index construction."""
    ii = np.ascontiguousarray(np.asarray(ii), dtype=np.int64)
    jj = np.ascontiguousarray(np.asarray(jj), dtype=np.int64)
    n = t1 - t0 + ii.shape[0]
    kx = np.zeros(n, dtype=np.int64)
    kk = np.zeros(n, dtype=np.int64)
    L = ctypes.c_int64
    K = lib().oracle_ba_index(_p(ii, L), _p(jj, L), ii.shape[0], t0, t1, _p(kx, L), _p(kk, L))
    return kx[:K], kk


def schur_pairs(ii, jj, t0, t1):
    """Pose-pair list (pi, pj) and row triplets of the reference's Schur enumeration."""
    ii = np.ascontiguousarray(np.asarray(ii), dtype=np.int64)
    jj = np.ascontiguousarray(np.asarray(jj), dtype=np.int64)
    L = ctypes.c_int64
    n = lib().oracle_schur_pairs(_p(ii, L), _p(jj, L), ii.shape[0], t0, t1, None, None, None)
    pi = np.zeros(n, dtype=np.int64)
    pj = np.zeros(n, dtype=np.int64)
    tr = np.zeros(3 * n, dtype=np.int64)
    lib().oracle_schur_pairs(_p(ii, L), _p(jj, L), ii.shape[0], t0, t1, _p(pi, L), _p(pj, L), _p(tr, L))
    return pi, pj, tr.reshape(-1, 3)


def accum_csr(ii, jj, t0, t1):
    """(ptr, idx): the edges grouped by source depth frame, as accum_cuda(., ii, kx) builds them."""
    ii = np.ascontiguousarray(np.asarray(ii), dtype=np.int64)
    jj = np.ascontiguousarray(np.asarray(jj), dtype=np.int64)
    L = ctypes.c_int64
    ptr = np.zeros(t1 - t0 + ii.shape[0] + 1, dtype=np.int64)
    idx = np.zeros(max(ii.shape[0], 1), dtype=np.int64)
    K = lib().oracle_accum_csr(_p(ii, L), _p(jj, L), ii.shape[0], t0, t1, _p(ptr, L), _p(idx, L))
    return ptr[:K + 1], idx[:ii.shape[0]]
