"""ORACLE - test infrastructure only.

Plain numpy / Python restatement of the data-parallel parts of the
negotiation bookkeeping (orthoroute_b200/bookkeeping.py and
orsp_bookkeeping.cu), following the reference line by line
(orthoroute/algorithms/manhattan/unified_pathfinder.py, "UPF"):

* node_owner         _rebuild_node_owner, committed via barrels (UPF:2785-2812)
* barrel_conflicts   _detect_barrel_conflicts (UPF:5520-5562)
* barrel_penalty     present[conflicts] += min(10 pres_fac, 100) (UPF:3852-3871)
* net_scores         the sums of _order_nets_by_difficulty (UPF:4406-4425) and
                     _build_hotset (UPF:5019-5071)

Pinned to the reference by tests/golden/golden_bookkeeping.npz.
"""
from __future__ import annotations

import numpy as np


def node_owner(N, nx, ny, paths, net_ids, keepouts=()):
    """paths: node lists in dict order; net_ids: their ids; keepouts:
    (z, x, y, id) in dict order."""
    owner = np.full(N, -1, np.int32)
    plane = nx * ny
    for path, nid in zip(paths, net_ids):
        for u, v in zip(path[:-1], path[1:]):
            zu, ru = divmod(int(u), plane)
            zv, rv = divmod(int(v), plane)
            if ru == rv and zu != zv:
                for z in range(min(zu, zv), max(zu, zv) + 1):
                    owner[z * plane + ru] = nid
    for z, x, y, nid in keepouts:
        if z <= 0:
            continue
        v = z * plane + y * nx + x
        if owner[v] == -1:
            owner[v] = nid
    return owner


def barrel_conflicts(indptr, indices, edge_lists, net_ids, owner):
    """(conflict edge ids in concatenation order, count)."""
    esrc = np.repeat(np.arange(len(indptr) - 1, dtype=np.int64), np.diff(indptr))
    e = np.concatenate([np.asarray(x, np.int64) for x in edge_lists]) if edge_lists else np.zeros(0, np.int64)
    ids = np.concatenate([np.full(len(x), i, np.int64) for x, i in zip(edge_lists, net_ids)]) if edge_lists else \
        np.zeros(0, np.int64)
    so, do = owner[esrc[e]], owner[np.asarray(indices)[e]]
    m = ((so != -1) & (so != ids)) | ((do != -1) & (do != ids))
    return e[m].astype(np.int32), int(m.sum())


def barrel_penalty(present, conflicts, pres_fac):
    out = present.copy()
    out[np.asarray(conflicts, np.int64)] += min(10.0 * pres_fac, 100.0)
    return out


def net_scores(edge_lists, present, capacity, history):
    """(congestion, impact, offender, hot edge count) with Python float sums."""
    over = np.maximum(0, present - capacity)
    hot = (over + 0.1 * history) > 0.5
    cong, imp, off = [], [], []
    for edges in edge_lists:
        cong.append(sum(float(over[e]) for e in edges) / max(1, len(edges)))
        imp.append(sum(float(over[e]) for e in edges if hot[e]))
        off.append(bool(any(hot[e] for e in edges)))
    return np.array(cong), np.array(imp), np.array(off, bool), int(hot.sum())
