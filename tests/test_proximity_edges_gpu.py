"""GPU proximity-edge construction against the reference's own edge lists and the oracle.

* tests/golden/proximity_edges.pt: edge lists the reference's FactorGraph.add_proximity_factors
  (vipe/slam/components/factor_graph.py:409-486) emitted (backend, frontend with prior edges and
  the factor cap, initialisation with cross-view edges) — reproduced exactly, through both
  vipe_b200.factor_graph_edges.proximity_edges and its drop-in add_proximity_factors method;
* larger seeded cases (backend windows of 256 and 1024 keyframes, prior edges, NaN and tied
  distances) against the CPU restatement oracle/edges.py, which the CPU tests pin to those
  same reference lists.
Integer work: compared with assert_array_equal.
"""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle.edges import proximity_edges as oracle_edges

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "proximity_edges.pt"


def _cases():
    return torch.load(GOLDEN, weights_only=False)["cases"]


@pytest.mark.parametrize("name", ["backend", "frontend", "init_cross_view"])
def test_matches_reference_edge_lists(name):
    from vipe_b200.factor_graph_edges import proximity_edges

    c = _cases()[name]
    ii, jj = proximity_edges(c["d"].cuda(), c["ii_exist"].cuda(), c["jj_exist"].cuda(), c["t0"], c["t1"], c["t"],
                             c["rad"], c["nms"], c["thresh"], c["max_factors"], c["cross_view"])
    np.testing.assert_array_equal(ii.cpu().numpy(), c["ii"].numpy())
    np.testing.assert_array_equal(jj.cpu().numpy(), c["jj"].numpy())


@pytest.mark.parametrize("name", ["backend", "frontend", "init_cross_view"])
def test_drop_in_method_on_a_graph(name):
    """The drop-in method on a stand-in graph that holds only what the reference method reads."""
    from vipe_b200.factor_graph_edges import add_proximity_factors

    c = _cases()[name]
    t, t0, t1 = c["t"], c["t0"], c["t1"]
    dm = torch.full((t, t), float("inf"), device="cuda")
    dm[t0:, t1:] = c["d"].view(t - t0, t - t1).cuda()

    class Buffer:
        n_frames = t

        @staticmethod
        def frame_distance_dense_disp(ii, jj, beta=0.3):
            return dm[ii, jj].unsqueeze(-1)

    class Graph:
        device = torch.device("cuda")
        buffer = Buffer()
        ii = c["ii_exist"].cuda()
        jj = c["jj_exist"].cuda()
        ii_inac = torch.zeros(0, dtype=torch.long, device="cuda")
        jj_inac = torch.zeros(0, dtype=torch.long, device="cuda")
        cross_view = c["cross_view"]
        max_factors = c["max_factors"]
        added = None

        def add_factors(self, ii, jj, remove=False):
            self.added = (ii, jj)

    g = Graph()
    add_proximity_factors(g, t0=t0, t1=t1, rad=c["rad"], nms=c["nms"], beta=0.3, thresh=c["thresh"])
    np.testing.assert_array_equal(g.added[0].cpu().numpy(), c["ii"].numpy())
    np.testing.assert_array_equal(g.added[1].cpu().numpy(), c["jj"].numpy())


def _distances(t, seed, loops):
    rng = np.random.default_rng(seed)
    pos = np.concatenate([[0.0], np.cumsum(rng.uniform(1.5, 4.0, t - 1))])
    d = np.abs(pos[:, None] - pos[None, :]) + rng.uniform(0.0, 1.0, (t, t))
    for _ in range(loops):
        i, j = sorted(rng.integers(0, t, 2).tolist())
        if j - i > 6:
            d[i, j] = d[j, i] = rng.uniform(2.0, 10.0)
    return d.astype(np.float32)


@pytest.mark.parametrize("t,t0,t1,nms,thresh,mf,prior", [(256, 0, 0, 3, 22.0, 16 * 256, 0),
                                                         (1024, 0, 0, 3, 22.0, 16 * 1024, 0),
                                                         (300, 200, 120, 1, 16.0, 900, 600)])
def test_large_cases_match_oracle(t, t0, t1, nms, thresh, mf, prior):
    from vipe_b200.factor_graph_edges import proximity_edges

    rng = np.random.default_rng(t + prior)
    dm = _distances(t, seed=t, loops=t // 8)
    d = dm[t0:, t1:].reshape(-1).copy()
    d[rng.integers(0, d.size, 5)] = np.nan  # NaN candidates: kept by the filter, visited last
    d[rng.integers(0, d.size, 40)] = 3.0  # exact ties: index order
    ie = rng.integers(t1, t, prior)
    je = np.clip(ie + rng.integers(-4, 5, prior), 0, t - 1)
    wi, wj = oracle_edges(d, ie, je, t0, t1, t, 2, nms, thresh, mf, False)
    gi, gj = proximity_edges(torch.from_numpy(d).cuda(), torch.from_numpy(ie).cuda(), torch.from_numpy(je).cuda(),
                             t0, t1, t, 2, nms, thresh, mf, False)
    np.testing.assert_array_equal(gi.cpu().numpy(), wi)
    np.testing.assert_array_equal(gj.cpu().numpy(), wj)
    assert len(wi) > 100
