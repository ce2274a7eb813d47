"""CPU restatement of the proximity-edge construction — TEST INFRASTRUCTURE ONLY.

Follows vipe/slam/components/factor_graph.py:431-486 (FactorGraph.add_proximity_factors,
after the frame distances are computed):
  * candidates (i, j), i in [t0, t), j in [t1, t), row-major, with distance d[k];
  * every existing edge (active, then inactive) suppresses the diamond
    |di| + |dj| <= max(min(|i - j| - 2, nms), 0) around it (d = inf);
  * candidates with i - rad < j or d > thresh are dropped;
  * the neighbourhood edges (i, j), (j, i) for j in [max(i - rad - 1, 0), i) are emitted
    first, i ascending (plus (i, i) first when cross_view), each suppressing its cell;
  * the remaining candidates are visited in ascending distance (a stable order here);
    one still at or below thresh is emitted as (i, j), (j, i) and suppresses its diamond,
    unless more than max_factors edges are already out, which ends the scan.
Returns the emitted (ii, jj) lists in order.
"""

from __future__ import annotations

import numpy as np


def proximity_edges(d, ii_exist, jj_exist, t0, t1, t, rad=2, nms=2, thresh=16.0, max_factors=48, cross_view=False):
    ni, nj = t - t0, t - t1
    d = np.array(d, dtype=np.float32).reshape(ni * nj).copy()

    def suppress(i, j):
        if t0 <= i < t and t1 <= j < t:
            d[(i - t0) * nj + (j - t1)] = np.inf

    def suppress_nms(i, j):
        r = max(min(abs(i - j) - 2, nms), 0)
        for di in range(-nms, nms + 1):
            for dj in range(-nms, nms + 1):
                if abs(di) + abs(dj) <= r:
                    suppress(i + di, j + dj)

    for i, j in zip(np.asarray(ii_exist).tolist(), np.asarray(jj_exist).tolist()):
        suppress_nms(int(i), int(j))
    ci = np.repeat(np.arange(t0, t), nj)
    cj = np.tile(np.arange(t1, t), ni)
    d[(ci - rad < cj) | (d > thresh)] = np.inf
    es = []
    for i in range(t0, t):
        if cross_view:
            es.append((i, i))
            suppress(i, i)
        for j in range(max(i - rad - 1, 0), i):
            es.append((i, j))
            es.append((j, i))
            suppress(i, j)
    order = np.argsort(d, kind="stable")
    for k in order.tolist():
        if d[k] > thresh:
            continue
        if len(es) > max_factors:
            break
        i, j = int(ci[k]), int(cj[k])
        es.append((i, j))
        es.append((j, i))
        suppress_nms(i, j)
    ii = np.array([e[0] for e in es], dtype=np.int64)
    jj = np.array([e[1] for e in es], dtype=np.int64)
    return ii, jj
