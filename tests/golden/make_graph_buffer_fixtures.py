"""Generates tests/golden/graph_buffer_fused_ba.pt from the reference's own Python BA code.

Run here, where the reference checkout exists (it does not exist on the GPU box):

    python tests/golden/make_graph_buffer_fixtures.py [/path/to/reference]

What it does.  The reference checks its fused BA against its generic torch
solver in tests/test_graph_buffer_fused_ba.py: two GraphBuffers are built by
that file's own helpers (`_make_video`, `_make_real_run_shaped_ba_inputs`), one
is solved by the generic solver (vipe/slam/ba/solver.py, terms.py, through
`GraphBuffer.bundle_adjustment`), the other by `GraphBuffer._fused_ba`
(buffer.py:364-489), which calls `slam_ext.ba_extended`, and the two buffers
must agree within 2e-4.  That test needs CUDA and the reference's compiled
extension.  This script runs every piece of it that is reference Python, on the
CPU, unchanged:
  * the test's helpers build both buffers (the test module's `torch.device`
    is pointed at the CPU; nothing else in it is touched);
  * the generic solver runs and its resulting poses, disparities and intrinsics
    are recorded;
  * `_fused_ba` runs with a recording `slam_ext` in place of the extension, so
    the exact arguments that GraphBuffer hands to `ba_extended` (layout
    conversion, sparse-track blending, eta, the 1/8 intrinsics, depth_active)
    are recorded.
tests/test_graph_buffer_fixtures_gpu.py then calls vipe_b200's
`slam_ext.ba_extended` with the recorded arguments on the GPU, applies the two
steps that follow the call in the reference (`disps.clamp_(min=0.001)` and the
intrinsics write-back, buffer.py:486-489 and :563) and compares with the generic
solver's result at the reference test's tolerance.

Robust kernels: config 0 with deterministic outlier flow is solved by the generic solver with
Huber, Tukey and GNC-TLS (the reference's fused path refuses robust kernels); the results go
to the "robust" entry and are held to vipe_slam_ba_extended_robust on the GPU.  The same
config 0 through the generic solver with the MEI camera (plain, and with Huber on the outlier
targets) goes to the "camera" entry (the fused path refuses non-pinhole buffers), and a two-view rig
(tests/_graph_buffer_golden.rig_problem) solved by GraphBuffer(n_views=2) to the "rig" entry.

The same is done for a third case built from config 0 (8 keyframes, 48x64 disparity,
26 edges, 2 iterations): GraphBuffer(384x512) is loaded with the config-0
workload, then both solvers run as above.  Its large inputs (targets, weights)
are regenerated on the GPU box by vipe_b200.workloads.ba_config0() and checked
there against the SHA-256 digests recorded here.

Import stubs (test infrastructure only): `omegaconf` and `rerun` are not
installed here and are replaced by minimal stand-ins; `vipe.ext` (the compiled
extension) is replaced by a package whose `lietorch_ext` evaluates the group
ops with the FP64 numpy oracle (oracle/lie.py) and returns them in the input
dtype, whose `slam_ext` records calls, and whose other members are empty; the
reference's own `vipe/ext/lietorch` and `vipe/ext/scatter.py` Python is used.
`vipe.streams.base` and `vipe.utils.visualization` (video I/O and drawing,
unused by BA) are stubbed.
"""

from __future__ import annotations

import hashlib
import importlib.util
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "graph_buffer_fused_ba.pt"


def sha256(t: torch.Tensor) -> str:
    return hashlib.sha256(t.detach().cpu().contiguous().numpy().tobytes()).hexdigest()


# ------------------------------------------------------------------ import stand-ins


class _Cfg(dict):
    """Attribute dict with .get, enough of omegaconf.DictConfig for GraphBuffer."""

    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as e:
            raise AttributeError(k) from e

    def __setattr__(self, k, v):
        self[k] = v


def _install_omegaconf():
    om = types.ModuleType("omegaconf")

    class OmegaConf:
        @staticmethod
        def create(d):
            return _Cfg(d)

        @staticmethod
        def has_resolver(name):
            return True

        @staticmethod
        def register_new_resolver(*a, **k):
            pass

    om.OmegaConf = OmegaConf
    om.DictConfig = _Cfg
    dc = types.ModuleType("omegaconf.dictconfig")
    dc.DictConfig = _Cfg
    om.dictconfig = dc
    sys.modules["omegaconf"] = om
    sys.modules["omegaconf.dictconfig"] = dc


def _lietorch_standin():
    import oracle.lie as ol

    m = types.ModuleType("lietorch_ext_oracle")

    def wrap(fn, n_group_args):
        def f(gid, *args):
            like = args[0]
            out = fn(gid, *[a.detach().double().cpu().numpy() for a in args])
            if isinstance(out, (list, tuple)):
                return [torch.as_tensor(np.asarray(o)).to(like.dtype) for o in out]
            return torch.as_tensor(np.asarray(out)).to(like.dtype)

        return f

    for name in ["expm", "logm", "inv", "mul", "adj", "adjT", "act", "act4", "as_matrix", "projector", "Jinv",
                 "expm_backward", "logm_backward", "inv_backward", "mul_backward", "adj_backward", "adjT_backward",
                 "act_backward", "act4_backward"]:
        setattr(m, name, wrap(getattr(ol, name), 0))
    return m


class RecordingSlamExt(types.ModuleType):
    def __init__(self):
        super().__init__("slam_ext_recorder")
        self.calls = []

    def ba_extended(self, *args):
        self.calls.append([a.detach().clone() if isinstance(a, torch.Tensor) else a for a in args])
        iters = int(args[12])
        return [None, None, torch.zeros(iters)]


def install_stubs(ref: Path):
    _install_omegaconf()
    sys.modules["rerun"] = types.ModuleType("rerun")
    if str(ref) not in sys.path:
        sys.path.insert(0, str(ref))
    import vipe  # noqa: F401  (the reference package; its __init__ only needs omegaconf)

    ext = types.ModuleType("vipe.ext")
    ext.__path__ = [str(ref / "vipe" / "ext")]
    ext.slam_ext = RecordingSlamExt()
    ext.lietorch_ext = _lietorch_standin()
    for name in ["scatter_ext", "utils_ext", "droid_net_ext", "corr_ext", "grounding_dino_ext"]:
        setattr(ext, name, types.ModuleType(name))
    sys.modules["vipe.ext"] = ext
    vipe.ext = ext

    sb = types.ModuleType("vipe.streams.base")

    class VideoFrame:  # only a type annotation target for BA
        pass

    sb.VideoFrame = VideoFrame
    sys.modules["vipe.streams.base"] = sb
    vis = types.ModuleType("vipe.utils.visualization")
    vis.POINTS_STENCIL = None
    vis.draw_lines_batch = vis.draw_points_batch = lambda *a, **k: None
    sys.modules["vipe.utils.visualization"] = vis
    return ext.slam_ext


def load_reference_test(ref: Path):
    """Imports tests/test_graph_buffer_fused_ba.py with its `torch.device` pointed at the CPU."""
    spec = importlib.util.spec_from_file_location("ref_test_graph_buffer_fused_ba",
                                                  ref / "tests" / "test_graph_buffer_fused_ba.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)

    class _TorchOnCPU(types.ModuleType):
        def __getattr__(self, k):
            return getattr(torch, k)

    proxy = _TorchOnCPU("torch_on_cpu")
    proxy.device = lambda *a, **k: torch.device("cpu")
    mod.torch = proxy
    return mod


# ------------------------------------------------------------------ cases


def state_of(video):
    return {"poses": video.poses.clone(), "disps": video.disps.clone(), "intrinsics": video.intrinsics.clone()}


def reference_test_case(mod, rec, *, motion_only, limited_disp, optimize_intrinsics, sparse):
    generic = mod._make_video(fused=False, sparse_tracks_enabled=sparse)
    fused = mod._make_video(fused=True, sparse_tracks_enabled=sparse)
    ba_inputs = mod._make_real_run_shaped_ba_inputs(generic)
    before = state_of(fused)
    kw = dict(motion_only=motion_only, limited_disp=limited_disp, optimize_intrinsics=optimize_intrinsics)
    mod._run_generic_bundle_adjustment(generic, ba_inputs, **kw)
    rec.calls.clear()
    assert mod._run_fused_bundle_adjustment(fused, ba_inputs, **kw)
    (args,) = rec.calls
    return {"kind": "reference_test", "args": args, "before": before, "generic": state_of(generic),
            "n_frames": 5, **kw}


def config0_case(rec):
    """Config 0 loaded into GraphBuffer (8 keyframes, 384x512 images -> 48x64 disparity)."""
    from vipe.slam.components.buffer import GraphBuffer
    from vipe.slam.components.sparse_tracks import DummySparseTracks
    from vipe.utils.cameras import CameraType

    from vipe_b200 import workloads as W

    p = W.ba_config0()
    N, ht, wd = p.disps.shape
    E = p.ii.shape[0]

    def make(fused):
        cfg = _Cfg({"dense_disp_alpha": float(p.alpha), "fused": fused, "intrinsics_damping_scale": 1.0,
                    "robust_kernel": None, "robust_kernel_threshold": 3.0, "gnc_mu_init": 1.0,
                    "gnc_mu_step": 3.0, "gnc_mu_max": 1.0e6, "gnc_n_mu_steps": 4, "gnc_gn_iters_per_mu": 6})
        v = GraphBuffer(height=8 * ht, width=8 * wd, n_views=1, buffer_size=N, init_disp=1.0, cross_view_idx=None,
                        ba_config=cfg, sparse_tracks=DummySparseTracks(n_views=1), camera_type=CameraType.PINHOLE,
                        device=torch.device("cpu"))
        v.n_frames = N
        v.tstamp[:N] = torch.arange(N)
        v.intrinsics[0, :4] = p.intrinsics * 8
        v.poses[:N] = p.poses
        v.disps[:N, 0] = p.disps
        v.disps_sens[:N, 0] = p.disps_sens
        return v

    target = p.targets.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
    weight = p.weights.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
    # eta = 0.2 * disp_damping[kx] + 1e-7 inside both solvers; kx = all frames here
    kx = torch.unique(torch.cat([torch.arange(p.t0, p.t1), p.ii]))
    assert torch.equal(kx, torch.arange(N))
    disp_damping = ((p.eta.double() - 1e-7) / 0.2).float()
    kw = dict(t0=p.t0, t1=p.t1, n_iters=p.iterations, pose_damping=float(p.lm), pose_ep=float(p.ep),
              motion_only=False, limited_disp=False, optimize_intrinsics=False, optimize_rig_rotation=False,
              verbose=False)
    generic = make(False)
    generic.bundle_adjustment(target=target.clone(), weight=weight.clone(), disp_damping=disp_damping.clone(),
                              ii=p.ii.clone(), jj=p.jj.clone(), **kw)
    fused = make(True)
    before = state_of(fused)
    rec.calls.clear()
    fused.bundle_adjustment(target=target.clone(), weight=weight.clone(), disp_damping=disp_damping.clone(),
                            ii=p.ii.clone(), jj=p.jj.clone(), **kw)
    (args,) = rec.calls
    # the recorded large inputs are exactly config 0's: store digests, regenerate on the GPU box
    assert torch.equal(args[4], p.targets) and torch.equal(args[5], p.weights)
    digests = {"targets": sha256(p.targets), "weights": sha256(p.weights)}
    args[4] = args[5] = None
    return {"kind": "config0", "args": args, "before": before, "generic": state_of(generic), "n_frames": N,
            "digests": digests, "motion_only": False, "limited_disp": False, "optimize_intrinsics": False}


ROBUST = {
    # name: (robust_kernel, threshold, n_iters, gnc settings)
    "huber": ("huber", 2.0, 3, {}),
    "tukey": ("tukey", 4.0, 3, {}),
    # GNC-TLS: two mu rounds of two iterations; mu 1 (soft weights), then min(3, 3) = mu_max
    # (the hard TLS indicator)
    "gnc_tls": ("gnc_tls", 3.0, 4, {"gnc_mu_init": 1.0, "gnc_mu_step": 3.0, "gnc_mu_max": 3.0,
                                    "gnc_n_mu_steps": 2, "gnc_gn_iters_per_mu": 2}),
}


CAMERA = {
    # name: (camera, k1, robust_kernel, threshold, n_iters)
    "mei": ("mei", 0.25, None, 1.0, 2),
    "mei_huber": ("mei", 0.6, "huber", 2.0, 3),
}


def camera_cases():
    """Config 0 through the reference's generic solver with the MEI camera (GraphBuffer with
    camera_type MEI: fx, fy, cx, cy of config 0 at full resolution and k1), plain and with
    Huber on the outlier targets.  The fused path refuses non-pinhole buffers
    (buffer.py:387-388)."""
    from vipe.slam.components.buffer import GraphBuffer
    from vipe.slam.components.sparse_tracks import DummySparseTracks
    from vipe.utils.cameras import CameraType

    sys.path.insert(0, str(ROOT / "tests"))
    from _graph_buffer_golden import with_outliers

    from vipe_b200 import workloads as W

    p = W.ba_config0()
    N, ht, wd = p.disps.shape
    E = p.ii.shape[0]
    weight = p.weights.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
    disp_damping = ((p.eta.double() - 1e-7) / 0.2).float()
    out = {}
    for name, (cam, k1, kernel, thr, n_iters) in CAMERA.items():
        targets = with_outliers(p.targets) if kernel else p.targets
        target = targets.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
        cfg = _Cfg({"dense_disp_alpha": float(p.alpha), "fused": False, "intrinsics_damping_scale": 1.0,
                    "robust_kernel": kernel, "robust_kernel_threshold": thr, "gnc_mu_init": 1.0,
                    "gnc_mu_step": 3.0, "gnc_mu_max": 1.0e6, "gnc_n_mu_steps": 4, "gnc_gn_iters_per_mu": 6})
        v = GraphBuffer(height=8 * ht, width=8 * wd, n_views=1, buffer_size=N, init_disp=1.0, cross_view_idx=None,
                        ba_config=cfg, sparse_tracks=DummySparseTracks(n_views=1), camera_type=CameraType.MEI,
                        device=torch.device("cpu"))
        v.n_frames = N
        v.tstamp[:N] = torch.arange(N)
        v.intrinsics[0, :4] = p.intrinsics * 8
        v.intrinsics[0, 4] = k1
        v.poses[:N] = p.poses
        v.disps[:N, 0] = p.disps
        v.disps_sens[:N, 0] = p.disps_sens
        v.bundle_adjustment(target=target.clone(), weight=weight.clone(), disp_damping=disp_damping.clone(),
                            ii=p.ii.clone(), jj=p.jj.clone(), t0=p.t0, t1=p.t1, n_iters=n_iters,
                            pose_damping=float(p.lm), pose_ep=float(p.ep), motion_only=False, limited_disp=False,
                            optimize_intrinsics=False, optimize_rig_rotation=False, verbose=False)
        out[name] = {"camera": cam, "k1": k1, "kernel": kernel, "threshold": thr, "iterations": n_iters,
                     "outliers": bool(kernel), "generic": state_of(v), "n_frames": N}
    return out


RIG = {
    # name: (outliers, robust_kernel, threshold, n_iters, per-view intrinsics + cross-view terms,
    #        rig rotation optimised from a perturbed initial rig, MEI k1 per view or None: pinhole)
    "rig": (False, None, 1.0, 2, False, False, None),
    "rig_huber": (True, "huber", 2.0, 3, False, False, None),
    "rig_views": (False, None, 1.0, 2, True, False, None),
    "rig_rot": (False, None, 1.0, 3, False, True, None),
    "rig_mei_views": (False, None, 1.0, 4, True, False, (0.15, 0.3)),
}


def rig_cases():
    """A two-view rig (tests/_graph_buffer_golden.rig_problem) solved by the reference's generic
    solver: GraphBuffer(n_views=2) with the rig extrinsics, expanded terms from
    expand_edge_multiview (the fused path refuses n_views > 1, buffer.py:387-388)."""
    from vipe.slam.components.buffer import GraphBuffer
    from vipe.slam.components.sparse_tracks import DummySparseTracks
    from vipe.utils.cameras import CameraType

    sys.path.insert(0, str(ROOT / "tests"))
    import _graph_buffer_golden as Gd

    out = {}
    for name, (outl, kernel, thr, n_iters, views, rig_rot, mei_k1) in RIG.items():
        r = Gd.rig_problem(outliers=outl, views=views, rig_error=rig_rot)
        N, V = r.N, r.V
        H, Wd = r.disps.shape[1:]
        cfg = _Cfg({"dense_disp_alpha": r.alpha, "fused": False, "intrinsics_damping_scale": 1.0,
                    "robust_kernel": kernel, "robust_kernel_threshold": thr, "gnc_mu_init": 1.0, "gnc_mu_step": 3.0,
                    "gnc_mu_max": 1.0e6, "gnc_n_mu_steps": 4, "gnc_gn_iters_per_mu": 6})
        v = GraphBuffer(height=8 * H, width=8 * Wd, n_views=V, buffer_size=N, init_disp=1.0, cross_view_idx=None,
                        ba_config=cfg, sparse_tracks=DummySparseTracks(n_views=V),
                        camera_type=CameraType.MEI if mei_k1 else CameraType.PINHOLE, device=torch.device("cpu"))
        v.n_frames = N
        v.tstamp[:N] = torch.arange(N)
        v.intrinsics[:, :4] = r.intrinsics * 8
        if mei_k1:
            v.intrinsics[:, 4] = torch.tensor(mei_k1)
        v.rig[:] = r.rig
        v.poses[:N] = r.poses
        v.disps[:N] = r.disps.reshape(N, V, H, Wd)
        v.disps_sens[:N] = r.disps_sens.reshape(N, V, H, Wd)
        # the expansion the generic solver makes must be the one the problem was built on
        pi, qi, di, pj, qj, dj = v.expand_edge_multiview(r.pi[::V], r.pj[::V])
        assert torch.equal(di, r.ii) and torch.equal(dj, r.jj)
        E = r.targets.shape[0]
        target = r.targets.permute(0, 2, 3, 1).reshape(E, H * Wd, 2).contiguous()
        weight = r.weights.permute(0, 2, 3, 1).reshape(E, H * Wd, 2).contiguous()
        disp_damping = r.disp_damping.repeat_interleave(V, 0).reshape(N * V, H, Wd)
        v.bundle_adjustment(target=target, weight=weight, disp_damping=disp_damping, ii=r.pi[::V].clone(),
                            jj=r.pj[::V].clone(), t0=r.t0, t1=r.t1, n_iters=n_iters, pose_damping=r.lm,
                            pose_ep=r.ep, motion_only=False, limited_disp=False, optimize_intrinsics=False,
                            optimize_rig_rotation=rig_rot, verbose=False)
        out[name] = {"outliers": outl, "kernel": kernel, "threshold": thr, "iterations": n_iters, "n_frames": N,
                     "views": views, "rig_rot": rig_rot, "rig": v.rig.clone(), "rig_before": r.rig.clone(),
                     "mei_k1": mei_k1,
                     "generic": {"poses": v.poses.clone(), "disps": v.disps.clone().reshape(-1, H, Wd)},
                     "before": {"poses": r.poses.clone()}}
    return out


def robust_cases():
    """Config 0 with deterministic outlier flow (tests/_graph_buffer_golden.with_outliers) solved
    by the reference's generic solver with each robust kernel (buffer.py:531-695; the fused path
    refuses robust kernels, buffer.py:541-545)."""
    from vipe.slam.components.buffer import GraphBuffer
    from vipe.slam.components.sparse_tracks import DummySparseTracks
    from vipe.utils.cameras import CameraType

    sys.path.insert(0, str(ROOT / "tests"))
    from _graph_buffer_golden import with_outliers

    from vipe_b200 import workloads as W

    p = W.ba_config0()
    N, ht, wd = p.disps.shape
    E = p.ii.shape[0]
    targets = with_outliers(p.targets)
    target = targets.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
    weight = p.weights.permute(0, 2, 3, 1).reshape(E, ht * wd, 2).contiguous()
    disp_damping = ((p.eta.double() - 1e-7) / 0.2).float()
    out = {}
    for name, (kernel, thr, n_iters, gnc) in ROBUST.items():
        cfg = _Cfg({"dense_disp_alpha": float(p.alpha), "fused": False, "intrinsics_damping_scale": 1.0,
                    "robust_kernel": kernel, "robust_kernel_threshold": thr, "gnc_mu_init": 1.0,
                    "gnc_mu_step": 3.0, "gnc_mu_max": 1.0e6, "gnc_n_mu_steps": 4, "gnc_gn_iters_per_mu": 6, **gnc})
        v = GraphBuffer(height=8 * ht, width=8 * wd, n_views=1, buffer_size=N, init_disp=1.0, cross_view_idx=None,
                        ba_config=cfg, sparse_tracks=DummySparseTracks(n_views=1), camera_type=CameraType.PINHOLE,
                        device=torch.device("cpu"))
        v.n_frames = N
        v.tstamp[:N] = torch.arange(N)
        v.intrinsics[0, :4] = p.intrinsics * 8
        v.poses[:N] = p.poses
        v.disps[:N, 0] = p.disps
        v.disps_sens[:N, 0] = p.disps_sens
        before = state_of(v)
        v.bundle_adjustment(target=target.clone(), weight=weight.clone(), disp_damping=disp_damping.clone(),
                            ii=p.ii.clone(), jj=p.jj.clone(), t0=p.t0, t1=p.t1, n_iters=n_iters,
                            pose_damping=float(p.lm), pose_ep=float(p.ep), motion_only=False, limited_disp=False,
                            optimize_intrinsics=False, optimize_rig_rotation=False, verbose=False)
        # the starting state is config 0's (the "config0" case's "before")
        assert torch.equal(before["poses"][:N], p.poses) and torch.equal(before["disps"][:N, 0], p.disps)
        out[name] = {"kernel": kernel, "threshold": thr, "iterations": n_iters, "gnc": gnc,
                     "generic": state_of(v), "n_frames": N}
    return out


def main(ref: Path):
    sys.path.insert(0, str(ROOT))
    rec = install_stubs(ref)
    mod = load_reference_test(ref)
    cases = {
        "intrinsics_limited_disp_sparse_tracks": reference_test_case(
            mod, rec, motion_only=False, limited_disp=True, optimize_intrinsics=True, sparse=True),
        "motion_only": reference_test_case(
            mod, rec, motion_only=True, limited_disp=False, optimize_intrinsics=False, sparse=False),
        "config0": config0_case(rec),
    }
    robust = robust_cases()
    camera = camera_cases()
    rig = rig_cases()
    torch.save({"cases": cases, "robust": robust, "camera": camera, "rig": rig, "torch": torch.__version__}, OUT)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    before = cases["config0"]["before"]["poses"]
    for k, c in {**cases, **{"robust_" + k: v for k, v in robust.items()},
                 **{"camera_" + k: v for k, v in camera.items()}, **{"rig_" + k: v for k, v in rig.items()}}.items():
        d = (c["generic"]["poses"] - c.get("before", {"poses": before})["poses"]).abs().max()
        print(f"  {k}: generic solver moved poses by {float(d):.3e}")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
