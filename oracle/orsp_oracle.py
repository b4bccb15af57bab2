"""ORACLE - test infrastructure only (the checker, never the product).

Python side of the oracle:

* ctypes bindings of orsp_oracle.c (heap Dijkstra, BFS ROI, path -> edges),
  the plain-C restatements of SimpleDijkstra.find_path_roi (UPF:1801-1887),
  ROIExtractor.extract_roi_bfs (UPF:1636-1734) and
  PathFinderRouter._path_to_edges (UPF:5463-5476);
* numpy restatements of EdgeAccountant (UPF:799-1068): the same float32 numpy
  expressions in the same order as the reference, so their bits are the
  reference's bits.

UPF = orthoroute/algorithms/manhattan/unified_pathfinder.py.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_LIB_PATH = _DIR / "liboracle.so"
_lib = None


def build_oracle(force: bool = False) -> Path:
    src = _DIR / "orsp_oracle.c"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(_DIR), "liboracle.so"], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build_oracle()
        lib = ctypes.CDLL(str(_LIB_PATH))
        P = ctypes.c_void_p
        i32 = ctypes.c_int32
        lib.oracle_dijkstra.argtypes = [i32, P, P, P, i32, P, P, i32, P, P, P, P, P, P, i32, P]
        lib.oracle_dijkstra.restype = ctypes.c_int
        lib.oracle_roi_bfs.argtypes = [i32, P, P, i32, i32, i32, i32, P]
        lib.oracle_roi_bfs.restype = i32
        lib.oracle_roi_bfs_keep.argtypes = [i32, P, P, i32, i32, i32, i32, P, i32, P]
        lib.oracle_roi_bfs_keep.restype = i32
        lib.oracle_path_to_edges.argtypes = [P, P, P, i32, P]
        lib.oracle_path_to_edges.restype = i32
        lib.oracle_batch_bbox.argtypes = [i32, P, P, P, i32, i32, i32, i32, P, P, P, P, i32, P]
        lib.oracle_batch_bbox.restype = ctypes.c_int
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def dijkstra(indptr, indices, cost, seeds, dst=-1, roi_map=None, seed_cost=None,
             targets=None, target_cost=None, path_cap=None):
    """Returns (path: np.ndarray int32 (empty = no path), dist float32[N],
    parent int32[N], best_target)."""
    lib = _load()
    indptr = _c(indptr, np.int32)
    indices = _c(indices, np.int32)
    cost = _c(cost, np.float32)
    N = indptr.shape[0] - 1
    seeds = _c(np.atleast_1d(seeds), np.int32)
    seed_cost = _c(seed_cost, np.float32)
    roi_map = _c(roi_map, np.int32)
    tmask = tcost = None
    if targets is not None:
        tmask = np.zeros(N, dtype=np.uint8)
        tcost = np.zeros(N, dtype=np.float64)
        targets = np.atleast_1d(targets)
        tc = np.zeros(len(targets)) if target_cost is None else np.asarray(target_cost, dtype=np.float64)
        for t, c in zip(targets, tc):  # later entries win, like a dict
            tmask[int(t)] = 1
            tcost[int(t)] = c
    dist = np.empty(N, dtype=np.float32)
    parent = np.empty(N, dtype=np.int32)
    cap = N + 1 if path_cap is None else path_cap
    path = np.empty(cap, dtype=np.int32)
    best = np.zeros(1, dtype=np.int32)
    rc = lib.oracle_dijkstra(N, _p(indptr), _p(indices), _p(cost), len(seeds), _p(seeds),
                             _p(seed_cost), int(dst), _p(roi_map), _p(tmask), _p(tcost),
                             _p(dist), _p(parent), _p(path), cap, _p(best))
    if rc < 0:
        raise RuntimeError(f"oracle_dijkstra failed ({rc})")
    return path[:rc].copy(), dist, parent, int(best[0])


def roi_bfs(indptr, indices, src, dst, max_depth, max_nodes=50_000, keep=None):
    """(roi_nodes int32[R], global_to_roi int32[N]); keep: extra must-keep
    nodes (the portal seeds of extract_roi_bfs, UPF:1700-1731)."""
    lib = _load()
    indptr = _c(indptr, np.int32)
    indices = _c(indices, np.int32)
    N = indptr.shape[0] - 1
    out = np.empty(N, dtype=np.int32)
    kp = _c(np.asarray([] if keep is None else keep, dtype=np.int32), np.int32)
    n = lib.oracle_roi_bfs_keep(N, _p(indptr), _p(indices), int(src), int(dst), int(max_depth),
                                int(max_nodes), _p(kp), int(kp.size), _p(out))
    if n < 0:
        raise RuntimeError("oracle_roi_bfs failed")
    roi = out[:n].copy()
    g2r = np.full(N, -1, dtype=np.int32)
    g2r[roi] = np.arange(n, dtype=np.int32)
    return roi, g2r


def path_to_edges(indptr, indices, path):
    lib = _load()
    indptr = _c(indptr, np.int32)
    indices = _c(indices, np.int32)
    path = _c(path, np.int32)
    out = np.empty(max(len(path) - 1, 1), dtype=np.int32)
    n = lib.oracle_path_to_edges(_p(indptr), _p(indices), _p(path), len(path), _p(out))
    return out[:n].copy()


def batch_bbox(indptr, indices, cost, nx, ny, nz, src, dst, bbox, path_cap):
    """Sequential box-ROI searches; returns (path_nodes[K, cap], path_len[K])."""
    lib = _load()
    indptr = _c(indptr, np.int32)
    indices = _c(indices, np.int32)
    cost = _c(cost, np.float32)
    src = _c(src, np.int32)
    dst = _c(dst, np.int32)
    bbox = _c(bbox, np.int32)
    K = len(src)
    nodes = np.zeros((K, path_cap), dtype=np.int32)
    lens = np.zeros(K, dtype=np.int32)
    rc = lib.oracle_batch_bbox(indptr.shape[0] - 1, _p(indptr), _p(indices), _p(cost), nx, ny, nz,
                               K, _p(src), _p(dst), _p(bbox), _p(nodes), path_cap, _p(lens))
    if rc < 0:
        raise RuntimeError("oracle_batch_bbox failed")
    return nodes, lens


# ---------------------------------------------------------------------------
# EdgeAccountant restatements (numpy float32, same expression order)
# ---------------------------------------------------------------------------

def update_costs(base, present_ema, capacity, history, pres_fac, hist_weight=1.0, add_jitter=True,
                 via_cost_multiplier=1.0, base_cost_weight=0.01, edge_layer=None,
                 layer_bias_per_layer=None, edge_kind=None):
    """EdgeAccountant.update_costs (UPF:973-1043)."""
    xp = np
    over = xp.maximum(0, present_ema - capacity)
    per_edge_bias = 1.0
    use_bias = edge_layer is not None and layer_bias_per_layer is not None and edge_kind is not None
    if use_bias:
        bias_factors = layer_bias_per_layer[edge_layer]
        per_edge_bias = xp.where(edge_kind == 0, bias_factors, 1.0)
    adjusted_base = base * via_cost_multiplier * base_cost_weight * per_edge_bias
    if use_bias:
        inverted_bias = xp.where(per_edge_bias != 0, 1.0 / xp.maximum(per_edge_bias, 0.5), 1.0)
        inverted_bias = xp.where(edge_kind == 0, inverted_bias, 1.0)
        present_term = (pres_fac * inverted_bias) * over
    else:
        present_term = pres_fac * over
    total = adjusted_base + present_term + hist_weight * history
    if add_jitter:
        E = len(total)
        jitter = xp.arange(E, dtype=xp.float32) % 9973
        jitter = jitter * 1e-6
        total += jitter
    return total


def update_present_ema(present, present_ema, beta=0.60):
    """EdgeAccountant.update_present_ema (UPF:963-971)."""
    return beta * present + (1.0 - beta) * present_ema


def update_history(history, present, capacity, gain, base_costs=None, history_cap_multiplier=10.0,
                   decay_factor=0.98):
    """EdgeAccountant.update_history (UPF:898-961) on the chosen present array."""
    history = history * decay_factor
    over = np.maximum(0, present - capacity)
    increment = gain * over
    if base_costs is not None:
        history_cap = history_cap_multiplier * base_costs
        increment = np.minimum(increment, history_cap)
    history += increment
    return history


def compute_overuse(present, capacity):
    """EdgeAccountant.compute_overuse (UPF:838-876), edge part."""
    edge_over = np.maximum(0, present - capacity)
    return int(edge_over.sum()), int((edge_over > 0).sum())


# ---------------------------------------------------------------------------
# Via pooling restatements (UPF:2678-2724, 3243-3387, 3448-3546, 5389-5461)
# ---------------------------------------------------------------------------

def via_edge_metadata(indptr, indices, nx, ny, nz):
    """(edge ids, x, y, z_lo, z_hi) of via edges (different layers), z range
    clamped to 1..nz-2, ascending edge id (_build_via_edge_metadata)."""
    indptr = np.asarray(indptr)
    indices = np.asarray(indices)
    plane = nx * ny
    src = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    zu = src // plane
    zv = indices // plane
    e = np.nonzero(zu != zv)[0]
    u = src[e]
    x = (u % plane) % nx
    y = (u % plane) // nx
    z_lo = np.clip(np.minimum(zu[e], zv[e]), 1, nz - 2)
    z_hi = np.clip(np.maximum(zu[e], zv[e]), 1, nz - 2)
    return e.astype(np.int32), x, y, z_lo, z_hi


def via_usage(paths, nx, ny, nz, col_use, seg_use):
    """Adds the via usage of node paths (_accumulate_via_usage_for_path)."""
    plane = nx * ny
    segz = max(nz - 2, 0)
    for path in paths:
        for u, v in zip(path, path[1:]):
            zu, ru = divmod(int(u), plane)
            zv, rv = divmod(int(v), plane)
            if ru != rv or zu == zv:
                continue
            x, y = ru % nx, ru // nx
            if col_use is not None:
                col_use[x, y] += 1
            if seg_use is not None:
                lo = max(1, min(min(zu, zv), nz - 2))
                hi = max(1, min(max(zu, zv), nz - 2))
                for z in range(lo, hi):
                    if 0 <= z - 1 < segz:
                        seg_use[x, y, z - 1] += 1


def via_present(col_use, col_cap, col_pres, seg_use, seg_cap, seg_pres, alpha=0.6, beta=0.4):
    """Smoothed via present costs and the z prefix (UPF:3622-3633)."""
    over = np.maximum(0, col_use - col_cap).astype(np.float32)
    col_pres = alpha * over + beta * col_pres
    over = np.maximum(0, seg_use - seg_cap).astype(np.float32)
    seg_pres = alpha * over + beta * seg_pres
    seg_prefix = np.cumsum(seg_pres, axis=2).astype(np.float32)
    return col_pres.astype(np.float32), seg_pres.astype(np.float32), seg_prefix


def via_penalties(total, meta, col_pres, seg_prefix, segz, layer_bias, pres_fac, col_weight=1.0,
                  seg_weight=1.0, k=0.20):
    """_apply_via_pooling_penalties, vectorised CPU path (UPF:3296-3380);
    layer_bias keeps its dtype (float32 or float64) like the reference's."""
    e, x, y, z_lo, z_hi = meta
    total = total.copy()
    pen = np.zeros(len(e), dtype=np.float32)
    if col_pres is not None:
        pen += col_weight * col_pres[x, y]
    if seg_prefix is not None:
        hi = z_hi - 2
        lo = z_lo - 2
        valid = z_hi > z_lo
        hv = (hi >= 0) & (hi < segz)
        lv = (lo >= 0) & (lo < segz)
        ph = np.zeros(len(e), dtype=np.float32)
        pl = np.zeros(len(e), dtype=np.float32)
        ph[hv] = seg_prefix[x[hv], y[hv], hi[hv]]
        pl[lv] = seg_prefix[x[lv], y[lv], lo[lv]]
        pen += seg_weight * ((ph - pl) * valid)
    if layer_bias is not None:
        sb = layer_bias[z_lo]
        db = layer_bias[z_hi]
        pen *= (1.0 - k * np.maximum(sb, 0.0)) * (1.0 + 0.5 * k * np.maximum(db, 0.0))
    m = pen > 0
    total[e[m]] += pres_fac * pen[m]
    return total


def via_hard_block(total, meta, col_use, col_cap, seg_use, seg_cap, segz):
    """_block_via_edges_with_collisions, CPU path (UPF:3499-3546)."""
    e, x, y, z_lo, z_hi = meta
    total = total.copy()
    for i in range(len(e)):
        xi, yi = int(x[i]), int(y[i])
        blocked = col_use is not None and col_use[xi, yi] >= col_cap[xi, yi]
        if not blocked and seg_use is not None:
            for z in range(int(z_lo[i]), int(z_hi[i])):
                if 0 <= z - 1 < segz and seg_use[xi, yi, z - 1] >= seg_cap[xi, yi, z - 1]:
                    blocked = True
                    break
        if blocked:
            total[e[i]] = np.float32("inf")
    return total
