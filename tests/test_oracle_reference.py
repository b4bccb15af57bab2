"""The oracle against the reference's own CPU code on seeded random inputs,
beyond the fixed golden vectors (CPU only; needs the reference source tree
and is skipped where it is absent): SimpleDijkstra.find_path_roi on random
lattices, costs and ROIs (integer costs, where the reference's float64 path
sums equal fp32), find_path_multisource_multisink with seed and portal
costs, ROIExtractor.extract_roi_bfs with random depths and node caps, the
EdgeAccountant updates with random parameters, the geometry emission
(_generate_geometry_from_paths) on random walks, and the negotiation
bookkeeping (_rebuild_node_owner, _detect_barrel_conflicts, _build_hotset,
_order_nets_by_difficulty) and the via pooling on random states."""
import logging
import os
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from orthoroute_b200.lattice import build_lattice

# the reference source tree, named by ORTHOROUTE_REFERENCE (skipped when unset)
REF = Path(os.environ.get("ORTHOROUTE_REFERENCE") or "/nonexistent")
pytestmark = pytest.mark.skipif(not (REF / "orthoroute").exists(), reason="reference source tree not available")


class _Graph:
    """The CSR attributes the reference's solver and ROI classes read."""

    def __init__(self, indptr, indices):
        self.indptr = indptr
        self.indices = indices
        self.base_costs = None
        self.xp = np


@pytest.fixture(scope="module")
def upf():
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.dont_write_bytecode = True
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    logging.disable(logging.CRITICAL)
    import orthoroute.algorithms.manhattan.unified_pathfinder as m

    return m


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_dijkstra_equals_reference_on_random_lattices(upf, seed):
    rng = np.random.default_rng(100 + seed)
    dims = [(int(rng.integers(3, 14)), int(rng.integers(3, 14)), int(rng.integers(1, 7))) for _ in range(3)]
    for nx, ny, nz in dims:
        lat = build_lattice(nx, ny, nz)
        g = _Graph(lat.indptr, lat.indices)
        solver = upf.SimpleDijkstra(g, lattice=None)
        ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
        cost = rng.integers(1, 8, size=lat.E).astype(np.float32)
        cost[lat.edge_kind == 1] = np.float32(rng.choice([2.0, 3.0, 5.0]))
        cost[rng.random(lat.E) < rng.choice([0.0, 0.05, 0.2])] = np.float32(np.inf)
        for j in range(10):
            s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
            if j % 2 == 0:
                roi = np.arange(lat.N, dtype=np.int32)
                g2r = np.arange(lat.N, dtype=np.int32)
            else:
                roi, g2r = ex.extract_roi_bfs(s, d, initial_radius=int(rng.integers(1, 10)))
            ref = upf.SimpleDijkstra.find_path_roi(solver, s, d, cost, roi, g2r)
            m = np.full(lat.N, -1, np.int32)
            m[np.asarray(roi)] = np.arange(len(roi), dtype=np.int32)
            p, *_ = O.dijkstra(lat.indptr, lat.indices, cost, [s], dst=d, roi_map=m)
            got = p.tolist() if len(p) > 1 else None
            assert got == (list(map(int, ref)) if ref else None), (nx, ny, nz, s, d)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed", [1, 2])
def test_roi_bfs_equals_reference_on_random_cases(upf, seed):
    rng = np.random.default_rng(200 + seed)
    lat = build_lattice(int(rng.integers(10, 30)), int(rng.integers(10, 30)), int(rng.integers(2, 6)))
    g = _Graph(lat.indptr, lat.indices)
    for _ in range(16):
        max_nodes = int(rng.choice([50_000, 800, 200, 60]))
        ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
        ex.max_roi_nodes = max_nodes
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        depth = int(rng.integers(1, 60))
        ref, _ = ex.extract_roi_bfs(s, d, initial_radius=depth)
        roi, g2r = O.roi_bfs(lat.indptr, lat.indices, s, d, min(depth, 150), max_nodes)
        assert np.array_equal(roi, np.asarray(ref, np.int32)), (s, d, depth, max_nodes)
        assert np.array_equal(g2r[roi], np.arange(len(roi)))


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_roi_bfs_with_portal_seeds_equals_reference(upf, seed):
    """extract_roi_bfs with portal_seeds: missing seeds appended as must-keep
    nodes, and kept through the truncation swap (UPF:1700-1731)."""
    rng = np.random.default_rng(250 + seed)
    lat = build_lattice(int(rng.integers(10, 30)), int(rng.integers(10, 30)), int(rng.integers(2, 6)))
    g = _Graph(lat.indptr, lat.indices)
    for _ in range(16):
        max_nodes = int(rng.choice([50_000, 800, 200, 60, 5]))
        ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
        ex.max_roi_nodes = max_nodes
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        depth = int(rng.integers(1, 30))
        # seeds near and far, with repeats and with src / dst among them
        seeds = [(int(v), float(rng.random())) for v in rng.choice(lat.N, size=int(rng.integers(1, 9)))]
        seeds += [(s, 0.0), seeds[0]]
        ref, _ = ex.extract_roi_bfs(s, d, initial_radius=depth, portal_seeds=seeds)
        roi, g2r = O.roi_bfs(lat.indptr, lat.indices, s, d, min(depth, 150), max_nodes,
                             keep=[n for n, _ in seeds])
        assert np.array_equal(roi, np.asarray(ref, np.int32)), (s, d, depth, max_nodes)


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_accounting_equals_reference_with_random_parameters(upf, seed):
    rng = np.random.default_rng(300 + seed)
    E, L = int(rng.integers(1000, 30000)), int(rng.integers(2, 10))
    base = rng.choice(np.array([0.4, 0.7, 1.0, 3.0], np.float32), size=E)
    present = rng.integers(0, 5, size=E).astype(np.float32)
    ema = (rng.random(E) * 3).astype(np.float32)
    cap = rng.choice(np.array([1.0, 2.0], np.float32), size=E)
    hist = (rng.random(E) * 5).astype(np.float32)
    edge_layer = rng.integers(0, L, size=E).astype(np.uint8)
    edge_kind = (rng.random(E) < 0.4).astype(np.uint8)
    bias = (0.3 + 1.7 * rng.random(L)).astype(np.float32)
    for _ in range(3):
        pf, hw = float(rng.choice([0.5, 1.5, 7.59375, 64.0])), float(rng.choice([1.0, 10.0, 12.0]))
        vm, bw = float(rng.choice([0.5, 1.0, 1.5])), float(rng.choice([0.01, 0.3, 1.0]))
        jit, ub = bool(rng.random() < 0.5), bool(rng.random() < 0.5)
        acc = upf.EdgeAccountant(E, use_gpu=False)
        acc.present_ema, acc.capacity, acc.history = ema.copy(), cap.copy(), hist.copy()
        acc.update_costs(base, pf, hw, add_jitter=jit, via_cost_multiplier=vm, base_cost_weight=bw,
                         edge_layer=edge_layer if ub else None, layer_bias_per_layer=bias if ub else None,
                         edge_kind=edge_kind if ub else None)
        got = O.update_costs(base, ema, cap, hist, pf, hw, add_jitter=jit, via_cost_multiplier=vm,
                             base_cost_weight=bw, edge_layer=edge_layer if ub else None,
                             layer_bias_per_layer=bias if ub else None, edge_kind=edge_kind if ub else None)
        assert np.array_equal(np.asarray(acc.total_cost, np.float32).view(np.uint32),
                              np.asarray(got, np.float32).view(np.uint32))
        gain, capm = float(rng.choice([0.25, 1.0, 1.2])), float(rng.choice([10.0, 15.0]))
        decay, use_base = float(rng.choice([0.98, 1.0])), bool(rng.random() < 0.5)
        acc = upf.EdgeAccountant(E, use_gpu=False)
        acc.present, acc.present_ema, acc.capacity, acc.history = present.copy(), ema.copy(), cap.copy(), hist.copy()
        acc.update_history(gain, base_costs=base if use_base else None, history_cap_multiplier=capm,
                           decay_factor=decay, use_raw_present=True)
        got = O.update_history(hist.copy(), present, cap, gain, base_costs=base if use_base else None,
                               history_cap_multiplier=capm, decay_factor=decay)
        assert np.array_equal(np.asarray(acc.history, np.float32).view(np.uint32),
                              np.asarray(got, np.float32).view(np.uint32))
    acc = upf.EdgeAccountant(E, use_gpu=False)
    acc.present, acc.present_ema = present.copy(), ema.copy()
    acc.update_present_ema(beta=0.4)
    assert np.array_equal(np.asarray(acc.present_ema, np.float32).view(np.uint32),
                          np.asarray(O.update_present_ema(present, ema, 0.4), np.float32).view(np.uint32))
    acc = upf.EdgeAccountant(E, use_gpu=False)
    acc.present, acc.capacity = present.copy(), cap.copy()
    assert tuple(acc.compute_overuse(None)) == O.compute_overuse(present, cap)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed", [1, 2])
def test_multisource_multisink_equals_reference(upf, seed):
    """find_path_multisource_multisink: seeds with start costs, targets with
    portal costs (sinks; the best total wins, ties to the target settled
    first), whole graph and BFS ROIs."""
    rng = np.random.default_rng(400 + seed)
    lat = build_lattice(int(rng.integers(6, 16)), int(rng.integers(6, 16)), int(rng.integers(2, 6)))
    g = _Graph(lat.indptr, lat.indices)
    solver = upf.SimpleDijkstra(g, lattice=None)
    ex = upf.ROIExtractor(g, use_gpu=False, lattice=None)
    cost = rng.integers(1, 6, size=lat.E).astype(np.float32)
    cost[rng.random(lat.E) < 0.05] = np.float32(np.inf)
    for i in range(16):
        ns, nt = int(rng.integers(1, 5)), int(rng.integers(1, 6))
        nodes = rng.choice(lat.N, size=ns + nt, replace=False)
        seeds, targets = nodes[:ns], nodes[ns:]
        scost = rng.integers(0, 4, size=ns) * 0.5
        tcost = rng.integers(0, 4, size=nt) * 0.25
        if i % 2:
            roi, g2r = ex.extract_roi_bfs(int(seeds[0]), int(targets[0]), initial_radius=int(rng.integers(2, 12)))
        else:
            roi = np.arange(lat.N, dtype=np.int32)
            g2r = np.arange(lat.N, dtype=np.int32)
        ref = solver.find_path_multisource_multisink(list(zip(seeds.tolist(), scost.tolist())),
                                                     list(zip(targets.tolist(), tcost.tolist())), cost, roi, g2r)
        m = np.full(lat.N, -1, np.int32)
        m[np.asarray(roi)] = np.arange(len(roi), dtype=np.int32)
        p, *_ = O.dijkstra(lat.indptr, lat.indices, cost, seeds, roi_map=m, seed_cost=scost.astype(np.float32),
                           targets=targets, target_cost=tcost)
        got = p.tolist() if len(p) > 1 else None
        assert got == (list(map(int, ref[0])) if ref else None), (i, seeds, targets)


def _random_path(rng, nx, ny, nz, dirs, n):
    """A walk on the lattice: mostly legal planar steps along each layer's
    axis and vias between adjacent layers, with a few illegal steps (a jump,
    a step across the layer's axis) for the reference's guards to drop."""
    x, y, z = int(rng.integers(0, nx)), int(rng.integers(0, ny)), int(rng.integers(0, nz))
    path = [z * nx * ny + y * nx + x]
    for _ in range(n):
        r = rng.random()
        if r < 0.2 and nz > 1:
            z2 = z + (1 if (z == 0 or (rng.random() < 0.5 and z < nz - 1)) else -1)
            z = min(max(z2, 0), nz - 1)
        elif r < 0.25:
            x = int(rng.integers(0, nx))  # a jump
        else:
            horizontal = dirs[z] == "h" if r < 0.95 else dirs[z] != "h"  # 5 %: across the axis
            step = 1 if rng.random() < 0.7 else -1
            if horizontal:
                x = min(max(x + step, 0), nx - 1)
            else:
                y = min(max(y + step, 0), ny - 1)
        node = z * nx * ny + y * nx + x
        if node != path[-1]:
            path.append(node)
    return path


@pytest.mark.parametrize("nz", [2, 4, 6])
def test_geometry_equals_reference_on_random_paths(upf, nz):
    """_generate_geometry_from_paths (with _segment_world / _via_world) on
    random walks, against the oracle's emission mapped to board coordinates
    as orthoroute_b200.geometry maps the device's."""
    import types

    from oracle.geometry import emit
    from orthoroute_b200.geometry import _quantize

    rng = np.random.default_rng(500 + nz)
    lat = upf.Lattice3D((10.3, 20.1, 18.7, 27.5), 0.4, nz)
    nx, ny = lat.x_steps, lat.y_steps
    dirs = [lat.get_legal_axis(z) for z in range(nz)]
    names = ["F.Cu"] + [f"In{i}.Cu" for i in range(1, nz - 1)] + ["B.Cu"]
    net_paths = {f"N{k}": _random_path(rng, nx, ny, nz, dirs, int(rng.integers(1, 60))) for k in range(40)}
    obj = types.SimpleNamespace(lattice=lat, net_paths=net_paths,
                                config=types.SimpleNamespace(layer_names=names, grid_pitch=0.4))
    obj._segment_world = types.MethodType(upf.PathFinderRouter._segment_world, obj)
    obj._via_world = types.MethodType(upf.PathFinderRouter._via_world, obj)
    ref_tracks, ref_vias = upf.PathFinderRouter._generate_geometry_from_paths(obj)

    gx0, gy0, plane = lat.geom.grid_min_x, lat.geom.grid_min_y, nx * ny

    def xy(node):
        r = int(node) % plane
        return (float(_quantize(gx0 + (r % nx) * 0.4, gx0, 0.4)), float(_quantize(gy0 + (r // nx) * 0.4, gy0, 0.4)))

    tracks, vias = [], []
    for name, (tr, vi) in zip(net_paths, emit(list(net_paths.values()), nx, ny, nz, dirs)):
        for a, b, z in tr:
            (x1, y1), (x2, y2) = xy(a), xy(b)
            tracks.append({"net": name, "layer": names[z], "x1": x1, "y1": y1, "x2": x2, "y2": y2, "width": 0.4 * 0.6})
        for n, z0, z1 in vi:
            x, y = xy(n)
            vias.append({"net": name, "x": x, "y": y, "from_layer": names[min(z0, z1)],
                         "to_layer": names[max(z0, z1)], "diameter": 0.25, "drill": 0.15})
    assert len(ref_vias) > 0 and (nz == 2 or len(ref_tracks) > 0)
    assert tracks == ref_tracks
    assert vias == ref_vias


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_hotset_and_difficulty_order_equal_reference(upf, seed):
    """_build_hotset over several iterations (freeze-clean counters, cooldown,
    the seeded 60/40 sample) and _order_nets_by_difficulty (seeded global
    random rotation), on random edge lists and congestion, against the host
    logic of orthoroute_b200.bookkeeping with the oracle's per-net scores."""
    import random
    import types

    from oracle.bookkeeping import net_scores
    from orthoroute_b200.bookkeeping import difficulty_order, select_hotset

    rng = np.random.default_rng(600 + seed)
    nx, ny, nz = 40, 30, 4
    E = 5000
    names = [f"N{k}" for k in range(int(rng.integers(150, 400)))]
    tasks = {n: (int(rng.integers(0, nx * ny * nz)), int(rng.integers(0, nx * ny * nz))) for n in names}
    net_to_edges = {n: sorted(set(rng.integers(0, E, size=int(rng.integers(1, 30))).tolist()))
                    for n in names if rng.random() < 0.9}
    edge_to_nets = {}
    for n, es in net_to_edges.items():
        for e in es:
            edge_to_nets.setdefault(e, set()).add(n)
    routed = {n for n in net_to_edges if rng.random() < 0.95}
    obj = types.SimpleNamespace(
        accounting=types.SimpleNamespace(use_gpu=False, present=None, capacity=np.ones(E, np.float32), history=None),
        config=types.SimpleNamespace(hotset_cap=int(rng.choice([64, 150, 512])), freeze_after_clean=3),
        net_paths={n: ([1, 2] if n in routed else []) for n in names}, _net_to_edges=net_to_edges,
        _edge_to_nets=edge_to_nets, iteration=0,
        lattice=types.SimpleNamespace(idx_to_coord=lambda i: (i % (nx * ny) % nx, i % (nx * ny) // nx, i // (nx * ny))))
    clean, last = {}, {}
    keys = list(net_to_edges)
    for it in range(1, 7):
        present = rng.integers(0, 3, size=E).astype(np.float32) * (rng.random(E) < (0.3 if it < 5 else 0.0))
        history = (rng.random(E) * 4).astype(np.float32) * (rng.random(E) < 0.1)
        obj.accounting.present, obj.accounting.history, obj.iteration = present, history, it
        ripped = set(rng.choice(names, size=3, replace=False).tolist()) if it % 2 else None
        ref = upf.PathFinderRouter._build_hotset(obj, tasks, ripped)
        cong, imp, off, hot = net_scores([net_to_edges[n] for n in keys], present, obj.accounting.capacity, history)
        got = select_hotset(tasks, keys, imp, off, hot, routed, it, clean, last, obj.config.hotset_cap, 3, ripped)
        assert got == ref, it
        assert clean == getattr(obj, "_net_clean_iters", {}) and last == getattr(obj, "_last_reroute_iter", {})
        random.seed(1000 * seed + it)
        ref_order = upf.PathFinderRouter._order_nets_by_difficulty(obj, tasks)
        random.seed(1000 * seed + it)
        got_order = difficulty_order(tasks, dict(zip(keys, (float(c) for c in cong))), nx, ny)
        assert got_order == ref_order, it


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_node_owner_and_barrel_conflicts_equal_reference(upf, seed):
    """_rebuild_node_owner (via barrels, last net wins; escape-via keepouts on
    free nodes, first entry wins) and _detect_barrel_conflicts on random
    overlapping paths, against the oracle's restatements."""
    import types

    import oracle.bookkeeping as OB

    rng = np.random.default_rng(700 + seed)
    nx, ny, nz = int(rng.integers(8, 20)), int(rng.integers(8, 20)), int(rng.integers(3, 7))
    lat = build_lattice(nx, ny, nz)
    plane = nx * ny
    paths = {}
    for k in range(int(rng.integers(10, 40))):
        u = int(rng.integers(0, lat.N))
        path = [u]
        for _ in range(int(rng.integers(0, 40))):
            nb = lat.indices[lat.indptr[u]:lat.indptr[u + 1]]
            if len(nb) == 0:
                break
            u = int(nb[rng.integers(0, len(nb))])
            path.append(u)
        paths[f"N{k}"] = path
    keep = {}
    for _ in range(int(rng.integers(0, 30))):
        keep[(int(rng.integers(0, nz)), int(rng.integers(0, nx)), int(rng.integers(0, ny)))] = \
            f"N{int(rng.integers(0, len(paths) + 3))}"
    obj = types.SimpleNamespace(
        lattice=types.SimpleNamespace(idx_to_coord=lambda i: (i % plane % nx, i % plane // nx, i // plane),
                                      node_idx=lambda x, y, z: z * plane + y * nx + x, num_nodes=lat.N, layers=nz),
        graph=types.SimpleNamespace(indptr=lat.indptr, indices=lat.indices), net_paths=paths,
        _via_keepouts_map=keep, node_owner=np.full(lat.N, -1, np.int32), net_id_map={}, next_net_id=0)
    for m in ("_get_net_id", "_ensure_edge_src_map", "_path_to_edges"):
        setattr(obj, m, types.MethodType(getattr(upf.PathFinderRouter, m), obj))
    upf.PathFinderRouter._rebuild_node_owner(obj)
    ref_owner = obj.node_owner.copy()
    ref_conf, ref_cnt = upf.PathFinderRouter._detect_barrel_conflicts(obj)
    ids = obj.net_id_map
    order = [n for n, p in paths.items() if len(p) >= 2]
    owner = OB.node_owner(lat.N, nx, ny, [paths[n] for n in order], [ids[n] for n in order],
                          [(z, x, y, ids[n]) for (z, x, y), n in keep.items()])
    assert np.array_equal(owner, ref_owner)
    edges = [O.path_to_edges(lat.indptr, lat.indices, np.asarray(paths[n], np.int32)) for n in order]
    conf, cnt = OB.barrel_conflicts(lat.indptr, lat.indices, edges, [ids[n] for n in order], owner)
    assert cnt == ref_cnt and np.array_equal(np.asarray(conf), np.asarray(ref_conf))
    assert (ref_owner >= 0).any() and (seed == 1 or ref_cnt > 0)


@pytest.mark.parametrize("seed,layers", [(1, 3), (2, 4), (3, 5)])
def test_via_pooling_equals_reference_on_random_states(upf, seed, layers):
    """Via usage, pooling penalties (float32 and float64 layer bias) and the
    hard block of full via columns / segments on the reference's own
    Lattice3D graph (blind and buried vias of every span), with random paths,
    capacities and present fields (tests/golden/make_golden.py gen_via with
    other seeds and sizes)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", Path(__file__).resolve().parent / "golden" /
                                                  "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    rng = np.random.default_rng(800 + seed)
    w, h = 0.4 * int(rng.integers(6, 14)), 0.4 * int(rng.integers(6, 14))
    lat = upf.Lattice3D((0.0, 0.0, w, h), 0.4, layers)
    graph = lat.build_graph(via_cost=0.7, use_gpu=False)
    g = mg.gen_via(upf, graph, lat, rng)
    nx, ny, nz = (int(v) for v in g["via_dims"])
    indptr, indices = np.asarray(graph.indptr, np.int32), np.asarray(graph.indices, np.int32)
    meta = O.via_edge_metadata(indptr, indices, nx, ny, nz)
    col = np.zeros((nx, ny), np.int64)
    seg = np.zeros((nx, ny, max(nz - 2, 0)), np.int64)
    O.via_usage([g[f"vpath{i}"] for i in range(int(g["npaths"]))], nx, ny, nz, col, seg)
    assert np.array_equal(col, g["col_use"]) and np.array_equal(seg, g["seg_use"])
    assert col.sum() > 0
    for tag in ("f32", "f64"):
        out = O.via_penalties(g["total0"], meta, g["col_pres"], g["seg_prefix"], nz - 2, g[f"bias_{tag}"], 2.25)
        assert np.array_equal(out.view(np.uint32), g[f"pen_{tag}"].view(np.uint32)), tag
    out = O.via_hard_block(g["total0"], meta, g["col_use"], g["col_cap"], g["seg_use"], g["seg_cap"], nz - 2)
    assert np.array_equal(out.view(np.uint32), g["blocked"].view(np.uint32))
