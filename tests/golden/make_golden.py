"""Generates the golden vectors in tests/golden/ by running the reference's own
CPU code (OrthoRoute, imported from its source tree: --ref or $ORTHOROUTE_REFERENCE).

Run from the repository root:
    python tests/golden/make_golden.py [--ref <OrthoRoute tree>]  (default: $ORTHOROUTE_REFERENCE)

Outputs (small .npz files, committed):
  golden_dijkstra.npz   SimpleDijkstra.find_path_roi (UPF:1801-1887) on
                        lattices with integer-valued costs (float64 path sums
                        are exact, so the reference's answer is the fp32 one)
                        and ROIs from ROIExtractor.extract_roi_bfs; plus the
                        reference's own Lattice3D graph (duplicated vias).
  golden_dijkstra_frac.npz  the same search with fractional costs (jitter-like),
                        where float64 and float32 sums may differ; the tests
                        report the agreement rate rather than require equality.
  golden_roi.npz        ROIExtractor.extract_roi_bfs (UPF:1636-1734), including
                        truncated ROIs (max_roi_nodes below the BFS size).
  golden_accounting.npz EdgeAccountant.update_costs / update_history /
                        update_present_ema / compute_overuse (UPF:799-1068).
  golden_path_edges.npz PathFinderRouter._path_to_edges (UPF:5463-5476).
  golden_via.npz        _accumulate_via_usage_for_path (UPF:2678-2724),
                        _apply_via_pooling_penalties (UPF:3243-3387, float32
                        and float64 layer bias) and
                        _block_via_edges_with_collisions (UPF:3448-3546) on the
                        reference's own blind/buried-via lattice.
UPF = orthoroute/algorithms/manhattan/unified_pathfinder.py.
"""
from __future__ import annotations

import argparse
import logging
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from orthoroute_b200.lattice import build_lattice  # noqa: E402


class _Graph:
    """Minimal CSRGraph stand-in (the attributes the reference classes read)."""

    def __init__(self, indptr, indices, base_costs=None):
        self.indptr = indptr
        self.indices = indices
        self.base_costs = base_costs
        self.xp = np


def import_reference(ref: str):
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref)
    logging.disable(logging.CRITICAL)
    import orthoroute.algorithms.manhattan.unified_pathfinder as upf  # noqa: E402

    return upf


def gen_dijkstra(upf, rng):
    cases = {}
    lats = [
        ("a", build_lattice(12, 10, 4)),
        ("b", build_lattice(9, 7, 6)),
        ("c", build_lattice(16, 16, 2)),
    ]
    out = {"names": []}
    k = 0
    for name, lat in lats:
        g = _Graph(lat.indptr, lat.indices)
        solver = upf.SimpleDijkstra(g, lattice=None)
        roi_ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
        cost = rng.integers(1, 6, size=lat.E).astype(np.float32)
        cost[lat.edge_kind == 1] = np.float32(3.0)
        blocked = rng.random(lat.E) < 0.05
        cost[blocked] = np.float32(np.inf)
        out[f"{name}_indptr"] = lat.indptr
        out[f"{name}_indices"] = lat.indices
        out[f"{name}_cost"] = cost
        out[f"{name}_dims"] = np.array([lat.nx, lat.ny, lat.nz], dtype=np.int32)
        for j in range(12):
            src, dst = rng.choice(lat.N, size=2, replace=False)
            if j % 3 == 0:
                roi = np.arange(lat.N, dtype=np.int32)
                g2r = np.arange(lat.N, dtype=np.int32)
            else:
                depth = int(rng.integers(2, 12))
                roi, g2r = roi_ex.extract_roi_bfs(int(src), int(dst), initial_radius=depth)
            path = solver.find_path_roi(int(src), int(dst), cost, roi, g2r)
            out[f"case{k}_lat"] = np.array([ord(name)], dtype=np.int32)
            out[f"case{k}_src"] = np.int32(src)
            out[f"case{k}_dst"] = np.int32(dst)
            out[f"case{k}_roi"] = np.asarray(roi, dtype=np.int32)
            out[f"case{k}_path"] = np.asarray(path if path else [], dtype=np.int32)
            k += 1
    out["ncases"] = np.int32(k)
    return out


def gen_reference_lattice(upf):
    """The reference's own Lattice3D.build_graph: planar edges on inner layers,
    blind/buried vias between all routing-layer pairs, duplicated via edges."""
    lat = upf.Lattice3D((0.0, 0.0, 4.0, 3.2), 0.4, 5)
    graph = lat.build_graph(via_cost=0.7, use_gpu=False)
    indptr = np.asarray(graph.indptr, dtype=np.int32)
    indices = np.asarray(graph.indices, dtype=np.int32)
    base = np.asarray(graph.base_costs, dtype=np.float32)
    return {
        "ref_dims": np.array([lat.x_steps, lat.y_steps, lat.layers], dtype=np.int32),
        "ref_indptr": indptr,
        "ref_indices": indices,
        "ref_base": base,
        "ref_edge_layer": np.asarray(graph.edge_layer, dtype=np.uint8),
        "ref_edge_kind": np.asarray(graph.edge_kind, dtype=np.uint8),
    }, graph, lat


def gen_dijkstra_frac(upf, rng):
    lat = build_lattice(14, 12, 4)
    g = _Graph(lat.indptr, lat.indices)
    solver = upf.SimpleDijkstra(g, lattice=None)
    base = np.where(lat.edge_kind == 1, np.float32(3.0), np.float32(1.0)).astype(np.float32)
    total = (base * np.float32(0.3) + np.arange(lat.E, dtype=np.float32) % 9973 * np.float32(1e-6)).astype(np.float32)
    noise = rng.integers(0, 4, size=lat.E).astype(np.float32) * np.float32(0.5)
    total = (total + noise).astype(np.float32)
    out = {"indptr": lat.indptr, "indices": lat.indices, "cost": total}
    srcs, dsts, paths = [], [], []
    for _ in range(40):
        s, d = rng.choice(lat.N, size=2, replace=False)
        roi = np.arange(lat.N, dtype=np.int32)
        p = solver.find_path_roi(int(s), int(d), total, roi, roi)
        srcs.append(s)
        dsts.append(d)
        paths.append(np.asarray(p if p else [], dtype=np.int32))
    out["src"] = np.asarray(srcs, dtype=np.int32)
    out["dst"] = np.asarray(dsts, dtype=np.int32)
    for i, p in enumerate(paths):
        out[f"path{i}"] = p
    return out


def gen_roi(upf, rng):
    lat = build_lattice(30, 24, 4)
    g = _Graph(lat.indptr, lat.indices)
    out = {"indptr": lat.indptr, "indices": lat.indices}
    k = 0
    for max_nodes in (50_000, 600, 250, 90):
        ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
        ex.max_roi_nodes = max_nodes
        for _ in range(6):
            s, d = rng.choice(lat.N, size=2, replace=False)
            depth = int(rng.integers(1, 40))
            roi, g2r = ex.extract_roi_bfs(int(s), int(d), initial_radius=depth)
            out[f"c{k}_args"] = np.array([s, d, depth, max_nodes], dtype=np.int64)
            out[f"c{k}_roi"] = np.asarray(roi, dtype=np.int32)
            k += 1
    # src == dst and adjacent src/dst
    ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
    for s, d, depth in ((5, 5, 3), (0, 1, 4)):
        roi, _ = ex.extract_roi_bfs(s, d, initial_radius=depth)
        out[f"c{k}_args"] = np.array([s, d, depth, 50_000], dtype=np.int64)
        out[f"c{k}_roi"] = np.asarray(roi, dtype=np.int32)
        k += 1
    out["ncases"] = np.int32(k)
    return out


def gen_accounting(upf, rng, ref_graph_arrays):
    E = 20_011
    L = 6
    out = {}
    base = rng.choice(np.array([0.4, 0.7, 1.0, 3.0], dtype=np.float32), size=E)
    present = rng.integers(0, 4, size=E).astype(np.float32)
    present[rng.random(E) < 0.01] += np.float32(2.5)  # barrel-penalty-like values
    ema = (rng.random(E) * 3).astype(np.float32)
    cap = np.ones(E, dtype=np.float32)
    hist = (rng.random(E) * 5).astype(np.float32)
    edge_layer = rng.integers(0, L, size=E).astype(np.uint8)
    edge_kind = (rng.random(E) < 0.4).astype(np.uint8)
    layer_bias = np.array([1.0, 1.3, 0.7, 1.8, 0.45, 1.0], dtype=np.float32)
    out.update(base=base, present=present, ema=ema, cap=cap, hist=hist, edge_layer=edge_layer,
               edge_kind=edge_kind, layer_bias=layer_bias)
    params = [
        # pres_fac, hist_weight, via_mult, base_w, jitter, use_bias
        (0.5, 12.0, 1.0, 0.3, True, False),
        (7.59375, 12.0, 0.5, 0.3, True, True),
        (1.0, 10.0, 1.5, 0.01, False, True),
        (64.0, 1.2, 1.0, 1.0, True, True),
    ]
    out["cost_params"] = np.array([[p[0], p[1], p[2], p[3], float(p[4]), float(p[5])] for p in params])
    for i, (pf, hw, vm, bw, jit, ub) in enumerate(params):
        acc = upf.EdgeAccountant(E, use_gpu=False)
        acc.present_ema = ema.copy()
        acc.capacity = cap.copy()
        acc.history = hist.copy()
        acc.update_costs(base, pf, hw, add_jitter=jit, via_cost_multiplier=vm, base_cost_weight=bw,
                         edge_layer=edge_layer if ub else None,
                         layer_bias_per_layer=layer_bias if ub else None,
                         edge_kind=edge_kind if ub else None)
        out[f"cost{i}"] = np.asarray(acc.total_cost, dtype=np.float32)
        assert out[f"cost{i}"].dtype == np.float32
    hparams = [(1.0, 15.0, 1.0, True), (1.2, 15.0, 0.98, True), (0.25, 10.0, 0.98, False)]
    out["hist_params"] = np.array([[a, b, c, float(d)] for a, b, c, d in hparams])
    for i, (gain, capm, decay, use_base) in enumerate(hparams):
        acc = upf.EdgeAccountant(E, use_gpu=False)
        acc.present = present.copy()
        acc.present_ema = ema.copy()
        acc.capacity = cap.copy()
        acc.history = hist.copy()
        acc.update_history(gain, base_costs=base if use_base else None, history_cap_multiplier=capm,
                           decay_factor=decay, use_raw_present=True)
        out[f"hist{i}"] = np.asarray(acc.history, dtype=np.float32)
    acc = upf.EdgeAccountant(E, use_gpu=False)
    acc.present = present.copy()
    acc.present_ema = ema.copy()
    acc.update_present_ema(beta=0.40)
    out["ema_out"] = np.asarray(acc.present_ema, dtype=np.float32)
    acc = upf.EdgeAccountant(E, use_gpu=False)
    ip = rng.integers(0, 3, size=E).astype(np.float32)
    acc.present = ip
    acc.capacity = cap.copy()
    out["over_present"] = ip
    out["overuse"] = np.array(acc.compute_overuse(None), dtype=np.int64)
    return out


def gen_path_edges(upf, graph, rng):
    """_path_to_edges on the reference lattice (duplicated via edges)."""
    indptr = np.asarray(graph.indptr, dtype=np.int32)
    indices = np.asarray(graph.indices, dtype=np.int32)
    N = len(indptr) - 1

    class _R:
        pass

    r = _R()
    r.graph = graph
    out = {}
    for k in range(20):
        # random walk along existing edges (plus one pair with no edge)
        u = int(rng.integers(0, N))
        while indptr[u + 1] == indptr[u]:
            u = int(rng.integers(0, N))
        path = [u]
        for _ in range(int(rng.integers(1, 25))):
            b, e = indptr[u], indptr[u + 1]
            if e == b:
                break
            u = int(indices[rng.integers(b, e)])
            path.append(u)
        if k % 5 == 4:
            path.append(int(rng.integers(0, N)))
        edges = upf.PathFinderRouter._path_to_edges(r, path)
        out[f"p{k}"] = np.asarray(path, dtype=np.int32)
        out[f"e{k}"] = np.asarray(edges, dtype=np.int32)
    out["n"] = np.int32(20)
    return out


def gen_via(upf, graph, lat, rng):
    """Via pooling on the reference's own lattice (blind/buried vias of every
    span): _accumulate_via_usage_for_path, _apply_via_pooling_penalties
    (float32 and float64 layer bias) and _block_via_edges_with_collisions,
    each called on a stub router holding just the attributes they read."""
    from types import SimpleNamespace

    Nx, Ny, Nz = lat.x_steps, lat.y_steps, lat.layers
    segz = Nz - 2
    indptr = np.asarray(graph.indptr, dtype=np.int32)
    indices = np.asarray(graph.indices, dtype=np.int32)
    N = len(indptr) - 1
    E = len(indices)

    def stub():
        st = SimpleNamespace()
        st.graph = graph
        st.lattice = lat
        st.config = SimpleNamespace(use_gpu=False, via_column_weight=1.0, via_segment_weight=1.0,
                                    via_hot_layer_discount=0.20)
        st._Nx, st._Ny, st._Nz, st._segZ = Nx, Ny, Nz, segz
        return st

    st = stub()
    upf.PathFinderRouter._identify_via_edges(st)
    upf.PathFinderRouter._build_via_edge_metadata(st)
    # random walks as committed paths
    paths = []
    for _ in range(60):
        u = int(rng.integers(0, N))
        path = [u]
        for _ in range(int(rng.integers(2, 30))):
            b, e = indptr[u], indptr[u + 1]
            if e == b:
                break
            u = int(indices[rng.integers(b, e)])
            path.append(u)
        paths.append(path)
    st.via_col_use = np.zeros((Nx, Ny), dtype=np.int16)
    st.via_seg_use = np.zeros((Nx, Ny, segz), dtype=np.int16)
    for pth in paths:
        upf.PathFinderRouter._accumulate_via_usage_for_path(st, pth, net_id=None)
    out = {"via_dims": np.array([Nx, Ny, Nz], dtype=np.int32), "npaths": np.int32(len(paths)),
           "col_use": st.via_col_use.copy(), "seg_use": st.via_seg_use.copy()}
    for i, pth in enumerate(paths):
        out[f"vpath{i}"] = np.asarray(pth, dtype=np.int32)
    col_cap = np.full((Nx, Ny), 4, dtype=np.int16)
    seg_cap = np.full((Nx, Ny, segz), 2, dtype=np.int8)
    col_cap[rng.random((Nx, Ny)) < 0.3] = 1
    seg_cap[rng.random((Nx, Ny, segz)) < 0.3] = 1
    out["col_cap"] = col_cap
    out["seg_cap"] = seg_cap
    # smoothing inputs / outputs are produced below with the reference's
    # inline expressions restated in oracle.via_present; the penalties use
    # random present fields so that every branch is exercised
    col_pres = (rng.random((Nx, Ny)) * 2).astype(np.float32)
    col_pres[rng.random((Nx, Ny)) < 0.5] = 0
    seg_pres = (rng.random((Nx, Ny, segz)) * 2).astype(np.float32)
    seg_prefix = np.cumsum(seg_pres, axis=2).astype(np.float32)
    total0 = (rng.random(E) * 3).astype(np.float32)
    out.update(col_pres=col_pres, seg_pres=seg_pres, seg_prefix=seg_prefix, total0=total0)
    for tag, bias in (("f32", np.array([1.0, 1.3, 0.8, 1.7, 1.1], dtype=np.float32)[:Nz]),
                      ("f64", np.array([1.0, 1.31, 0.77, 1.62, 1.05], dtype=np.float64)[:Nz])):
        st2 = stub()
        st2._via_edge_metadata = st._via_edge_metadata
        st2.via_col_pres = col_pres.copy()
        st2.via_seg_pres = seg_pres.copy()
        st2.via_seg_prefix = seg_prefix.copy()
        st2.layer_bias = bias
        st2.accounting = SimpleNamespace(total_cost=total0.copy(), use_gpu=False)
        upf.PathFinderRouter._apply_via_pooling_penalties(st2, 2.25)
        out[f"bias_{tag}"] = bias
        out[f"pen_{tag}"] = np.asarray(st2.accounting.total_cost, dtype=np.float32)
    st3 = stub()
    st3._via_edge_metadata = st._via_edge_metadata
    st3.via_col_use = st.via_col_use.copy()
    st3.via_col_cap = col_cap
    st3.via_seg_use = st.via_seg_use.copy()
    st3.via_seg_cap = seg_cap
    st3.accounting = SimpleNamespace(total_cost=total0.copy(), use_gpu=False)
    upf.PathFinderRouter._block_via_edges_with_collisions(st3)
    out["blocked"] = np.asarray(st3.accounting.total_cost, dtype=np.float32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ORTHOROUTE_REFERENCE"),
                    required=not os.environ.get("ORTHOROUTE_REFERENCE"),
                    help="OrthoRoute source tree (default: $ORTHOROUTE_REFERENCE)")
    args = ap.parse_args()
    upf = import_reference(args.ref)
    rng = np.random.default_rng(20261203)
    d = gen_dijkstra(upf, rng)
    ref_arrays, graph, _ = gen_reference_lattice(upf)
    # searches on the reference's own lattice (integer-valued costs)
    g = _Graph(ref_arrays["ref_indptr"], ref_arrays["ref_indices"])
    solver = upf.SimpleDijkstra(g, lattice=None)
    N = len(ref_arrays["ref_indptr"]) - 1
    E = len(ref_arrays["ref_indices"])
    rcost = rng.integers(1, 4, size=E).astype(np.float32)
    d.update(ref_arrays)
    d["ref_cost"] = rcost
    nref = 0
    for _ in range(15):
        s, t = rng.choice(N, size=2, replace=False)
        roi = np.arange(N, dtype=np.int32)
        p = solver.find_path_roi(int(s), int(t), rcost, roi, roi)
        d[f"ref{nref}_st"] = np.array([s, t], dtype=np.int32)
        d[f"ref{nref}_path"] = np.asarray(p if p else [], dtype=np.int32)
        nref += 1
    d["nref"] = np.int32(nref)
    np.savez_compressed(HERE / "golden_dijkstra.npz", **d)
    np.savez_compressed(HERE / "golden_dijkstra_frac.npz", **gen_dijkstra_frac(upf, rng))
    np.savez_compressed(HERE / "golden_roi.npz", **gen_roi(upf, rng))
    np.savez_compressed(HERE / "golden_accounting.npz", **gen_accounting(upf, rng, ref_arrays))
    np.savez_compressed(HERE / "golden_path_edges.npz", **gen_path_edges(upf, graph, rng))
    ref_lat = upf.Lattice3D((0.0, 0.0, 4.0, 3.2), 0.4, 5)
    np.savez_compressed(HERE / "golden_via.npz", **gen_via(upf, graph, ref_lat, np.random.default_rng(77)))
    for f in sorted(HERE.glob("golden_*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
