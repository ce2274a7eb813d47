"""Generates tests/golden/proximity_edges.pt from the reference's own edge construction.

Run here, where the reference checkout exists (it does not exist on the GPU box):

    python tests/golden/make_proximity_fixtures.py [/path/to/reference]

It calls the reference's FactorGraph.add_proximity_factors
(vipe/slam/components/factor_graph.py:409-486) unchanged, on a stand-in `self`
that holds only what the method reads: the buffer's frame count and its
frame_distance_dense_disp (returning a fixed distance matrix), the active and
inactive edge lists, cross_view, max_factors and a recording add_factors.  The
recorded edge lists, with the inputs, are what vipe_b200's GPU edge
construction must reproduce exactly (tests/test_proximity_edges_gpu.py), and
what pins the CPU restatement oracle/edges.py (tests/test_proximity_edges.py).

Scenarios (parameters from configs/slam/default.yaml and the callers
frontend.py:89-96, :135 and backend.py:79-94):
  backend    t = 64, t0 = t1 = 0, rad 2, nms 3, thresh 22, max_factors 16 t, no prior edges;
  frontend   t = 40, t0 = 35, t1 = 15, rad 2, nms 1, thresh 16, max_factors 48, with
             active and inactive edges (the cap ends the scan);
  init       t = 24, t0 = t1 = 0, rad 2, nms 2, thresh 16, cross_view, a few prior edges.
Distances: |i - j| times a per-frame speed plus noise, with low-distance loop pairs,
seeded, float32, no ties.
"""

from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
OUT = HERE / "proximity_edges.pt"


def distances(t, seed, loops=6):
    rng = np.random.default_rng(seed)
    speed = rng.uniform(1.5, 4.0, t)
    pos = np.concatenate([[0.0], np.cumsum(speed[1:])])
    d = np.abs(pos[:, None] - pos[None, :]) + rng.uniform(0.0, 1.0, (t, t))
    for _ in range(loops):  # revisits: far-apart frames that see the same place
        i, j = sorted(rng.integers(0, t, 2).tolist())
        if j - i > 6:
            d[i, j] = d[j, i] = rng.uniform(2.0, 10.0)
    return torch.from_numpy(d.astype(np.float32))


class StubGraph:
    def __init__(self, t, dmat, ii, jj, ii_inac, jj_inac, cross_view, max_factors):
        self.device = torch.device("cpu")
        dm = dmat

        class Buffer:
            n_frames = t

            @staticmethod
            def frame_distance_dense_disp(ii_, jj_, beta=0.3):
                return dm[ii_, jj_].unsqueeze(-1)

        self.buffer = Buffer()
        self.ii = torch.as_tensor(ii, dtype=torch.long)
        self.jj = torch.as_tensor(jj, dtype=torch.long)
        self.ii_inac = torch.as_tensor(ii_inac, dtype=torch.long)
        self.jj_inac = torch.as_tensor(jj_inac, dtype=torch.long)
        self.cross_view = cross_view
        self.max_factors = max_factors
        self.added = None

    def add_factors(self, ii, jj, remove=False):
        self.added = (ii.clone(), jj.clone())


def run_case(FactorGraph, t, t0, t1, rad, nms, thresh, max_factors, cross_view, ii, jj, ii_inac, jj_inac, seed):
    dmat = distances(t, seed)
    g = StubGraph(t, dmat, ii, jj, ii_inac, jj_inac, cross_view, max_factors)
    FactorGraph.add_proximity_factors(g, t0=t0, t1=t1, rad=rad, nms=nms, beta=0.3, thresh=thresh, remove=False)
    ix = torch.arange(t0, t)
    jx = torch.arange(t1, t)
    cand = dmat[ix[:, None], jx[None, :]].reshape(-1)
    return {"d": cand, "t": t, "t0": t0, "t1": t1, "rad": rad, "nms": nms, "thresh": thresh,
            "max_factors": max_factors, "cross_view": cross_view,
            "ii_exist": torch.cat([g.ii, g.ii_inac]), "jj_exist": torch.cat([g.jj, g.jj_inac]),
            "ii": g.added[0], "jj": g.added[1]}


def main(ref: Path):
    sys.path.insert(0, str(HERE))
    sys.path.insert(0, str(HERE.parents[1]))
    import make_graph_buffer_fixtures as M

    M.install_stubs(ref)
    from vipe.slam.components.factor_graph import FactorGraph

    band = [(i, j) for i in range(20, 38) for j in range(20, 38) if 0 < abs(i - j) <= 2]
    inac = [(i, j) for i in range(8, 22) for j in range(8, 22) if 0 < abs(i - j) <= 1]
    cases = {
        "backend": run_case(FactorGraph, 64, 0, 0, 2, 3, 22.0, 16 * 64, False, [], [], [], [], seed=2001),
        "frontend": run_case(FactorGraph, 40, 35, 15, 2, 1, 16.0, 48, False, [e[0] for e in band],
                             [e[1] for e in band], [e[0] for e in inac], [e[1] for e in inac], seed=2002),
        "init_cross_view": run_case(FactorGraph, 24, 0, 0, 2, 2, 16.0, 16 * 24, True, [3, 4, 10], [4, 3, 16],
                                    [], [], seed=2003),
    }
    torch.save({"cases": cases}, OUT)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    for k, c in cases.items():
        print(f"  {k}: {int(c['d'].numel())} candidates -> {int(c['ii'].numel())} edges")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
