"""The proximity-edge oracle (oracle/edges.py) against the reference's own add_proximity_factors.

tests/golden/proximity_edges.pt holds the edge lists that the reference's
FactorGraph.add_proximity_factors (vipe/slam/components/factor_graph.py:409-486)
emitted for three scenarios (backend, frontend with prior edges and the factor cap,
initialisation with cross-view edges), recorded by tests/golden/make_proximity_fixtures.py.
The CPU restatement must give the same lists, in the same order, integer for integer.
"""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle.edges import proximity_edges

GOLDEN = Path(__file__).resolve().parent / "golden" / "proximity_edges.pt"


def _cases():
    return torch.load(GOLDEN, weights_only=False)["cases"]


@pytest.mark.parametrize("name", ["backend", "frontend", "init_cross_view"])
def test_oracle_matches_reference_edge_lists(name):
    c = _cases()[name]
    ii, jj = proximity_edges(c["d"].numpy(), c["ii_exist"].numpy(), c["jj_exist"].numpy(), c["t0"], c["t1"], c["t"],
                             c["rad"], c["nms"], c["thresh"], c["max_factors"], c["cross_view"])
    np.testing.assert_array_equal(ii, c["ii"].numpy())
    np.testing.assert_array_equal(jj, c["jj"].numpy())
    assert len(ii) > 40
