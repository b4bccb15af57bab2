"""CUDA path (through the C ABI) against the oracle and the reference's golden
vectors.  Integer / index results must be identical; fp32 results bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as O  # noqa: E402
from orthoroute_b200 import _lib  # noqa: E402
from orthoroute_b200.accounting import DeviceEdgeAccountant  # noqa: E402
from orthoroute_b200.lattice import build_lattice, random_boxes, uniform_weights  # noqa: E402
from orthoroute_b200.solver import DeviceGraph, GpuSolver  # noqa: E402


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


def cuda(a, dt=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dt is not None:
        t = t.to(dt)
    return t.cuda()


# ---------------------------------------------------------------- accounting
def test_update_costs_bit_exact(golden):
    g = golden("golden_accounting.npz")
    E = len(g["base"])
    acc = DeviceEdgeAccountant(E)
    acc.present_ema.copy_(cuda(g["ema"]))
    acc.capacity.copy_(cuda(g["cap"]))
    acc.history.copy_(cuda(g["hist"]))
    for i, row in enumerate(g["cost_params"]):
        pf, hw, vm, bw, jit, ub = row
        acc.update_costs(g["base"], float(pf), float(hw), add_jitter=bool(jit), via_cost_multiplier=float(vm),
                         base_cost_weight=float(bw), edge_layer=g["edge_layer"] if ub else None,
                         layer_bias_per_layer=g["layer_bias"] if ub else None,
                         edge_kind=g["edge_kind"] if ub else None)
        assert np.array_equal(_bits(acc.total_cost.cpu().numpy()), _bits(g[f"cost{i}"])), f"param set {i}"


def test_history_ema_overuse_bit_exact(golden):
    g = golden("golden_accounting.npz")
    E = len(g["base"])
    for i, row in enumerate(g["hist_params"]):
        gain, capm, decay, use_base = row
        acc = DeviceEdgeAccountant(E)
        acc.present.copy_(cuda(g["present"]))
        acc.capacity.copy_(cuda(g["cap"]))
        acc.history.copy_(cuda(g["hist"]))
        acc.update_history(float(gain), base_costs=g["base"] if use_base else None,
                           history_cap_multiplier=float(capm), decay_factor=float(decay), use_raw_present=True)
        assert np.array_equal(_bits(acc.history.cpu().numpy()), _bits(g[f"hist{i}"]))
    acc = DeviceEdgeAccountant(E)
    acc.present.copy_(cuda(g["present"]))
    acc.present_ema.copy_(cuda(g["ema"]))
    acc.update_present_ema(beta=0.40)
    assert np.array_equal(_bits(acc.present_ema.cpu().numpy()), _bits(g["ema_out"]))
    acc = DeviceEdgeAccountant(E)
    acc.present.copy_(cuda(g["over_present"]))
    assert acc.compute_overuse() == tuple(int(v) for v in g["overuse"])


def test_update_costs_jitter_past_2_24():
    E = (1 << 24) + 40_000
    rng = np.random.default_rng(0)
    base = rng.choice(np.array([1.0, 3.0], np.float32), size=E)
    ema = rng.integers(0, 3, size=E).astype(np.float32)
    hist = (rng.random(E) * 2).astype(np.float32)
    cap = np.ones(E, np.float32)
    ref = O.update_costs(base, ema, cap, hist, 3.375, 1.2, add_jitter=True, base_cost_weight=0.3)
    acc = DeviceEdgeAccountant(E)
    acc.present_ema.copy_(cuda(ema))
    acc.history.copy_(cuda(hist))
    acc.update_costs(base, 3.375, 1.2, add_jitter=True, base_cost_weight=0.3)
    assert np.array_equal(_bits(acc.total_cost.cpu().numpy()), _bits(ref))


def test_commit_clear_semantics():
    acc = DeviceEdgeAccountant(16)
    acc.commit_path([1, 2, 2, 5])
    acc.clear_path([2, 7])  # 7 was never committed: stays 0
    u = acc.usage.cpu().numpy()
    assert u.tolist()[:8] == [0, 1, 1, 0, 0, 1, 0, 0]
    assert acc.present.cpu().numpy().tolist()[:8] == [0, 1, 1, 0, 0, 1, 0, 0]
    assert acc.verify_present_matches_canonical()
    assert acc.canonical == {1: 1, 2: 1, 5: 1}


# ------------------------------------------------------------------- search
def test_sssp_reference_golden_paths(golden):
    g = golden("golden_dijkstra.npz")
    graphs = {}
    for name in ("a", "b", "c"):
        ip, ix = g[f"{name}_indptr"], g[f"{name}_indices"]
        graphs[ord(name)] = (GpuSolver(DeviceGraph(ip, ix)), g[f"{name}_cost"])
    for k in range(int(g["ncases"])):
        solver, cost = graphs[int(g[f"case{k}_lat"][0])]
        roi = g[f"case{k}_roi"]
        g2r = np.full(solver.N, -1, np.int32)
        g2r[roi] = np.arange(len(roi), dtype=np.int32)
        p = solver.find_path_roi_gpu(int(g[f"case{k}_src"]), int(g[f"case{k}_dst"]), cost, roi, g2r)
        ref = g[f"case{k}_path"].tolist()
        assert (p or []) == ref, f"case {k}"


def test_sssp_reference_lattice_duplicate_vias(golden):
    g = golden("golden_dijkstra.npz")
    solver = GpuSolver(DeviceGraph(g["ref_indptr"], g["ref_indices"]))
    cost = g["ref_cost"]
    N = solver.N
    roi = np.arange(N, dtype=np.int32)
    for k in range(int(g["nref"])):
        s, d = (int(v) for v in g[f"ref{k}_st"])
        p = solver.find_path_roi_gpu(s, d, cost, roi, roi)
        assert (p or []) == g[f"ref{k}_path"].tolist()


@pytest.mark.parametrize("impl", ["lattice16", "lattice32", "lattice16-rounds", "generic"])
@pytest.mark.parametrize("shape,blocked,planar", [((60, 50, 6), 0.05, "all"), ((33, 17, 12), 0.0, "all"),
                                                  ((128, 96, 4), 0.03, "all"), ((45, 70, 6), 0.02, "inner")])
def test_sssp_full_distances_bit_exact(shape, blocked, planar, impl, monkeypatch):
    """Full searches, both implementations (tile sweeps on the lattice, generic
    near-far) and both tile sizes, bit-identical to the oracle."""
    monkeypatch.setenv("ORSP_SSSP_IMPL", "generic" if impl == "generic" else "auto")
    monkeypatch.setenv("ORSP_LAT_TILE", "32" if impl == "lattice32" else "16")
    monkeypatch.setenv("ORSP_LAT_ASYNC", "0" if impl.endswith("rounds") else "1")
    lat = build_lattice(*shape, planar=planar)
    w = uniform_weights(lat, seed=sum(shape), blocked_frac=blocked)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    rng = np.random.default_rng(7)
    for s in rng.choice(lat.N, size=3, replace=False):
        _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(s)])
        for delta in (0.37, 2.0, 1e4):
            dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
            st, _, rounds = dg.sssp(wt, int(s), -1, delta=delta, dist_out=dist)
            assert st == _lib.ORSP_OK
            assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), f"src {s} delta {delta}"


def test_sssp_paths_random_targets_and_rois():
    lat = build_lattice(70, 40, 6)
    w = uniform_weights(lat, seed=11, blocked_frac=0.04)
    dg = DeviceGraph.from_lattice(lat)
    solver = GpuSolver(dg)
    rng = np.random.default_rng(3)
    for i in range(40):
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        if i % 2:
            roi, g2r = O.roi_bfs(lat.indptr, lat.indices, s, d, int(rng.integers(3, 60)), 50_000)
        else:
            roi = np.arange(lat.N, dtype=np.int32)
            g2r = roi
        ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=None if i % 2 == 0 else g2r)
        got = solver.find_path_roi_gpu(s, d, w, roi, g2r)
        assert (got or []) == (ref.tolist() if len(ref) > 1 else [])


def test_sssp_edge_cases():
    lat = build_lattice(10, 8, 4)
    w = np.ones(lat.E, np.float32)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    # src == dst: single node, reference returns None
    st, p, _ = dg.sssp(wt, 5, 5)
    assert st == _lib.ORSP_NO_PATH
    # unreachable: block every edge into node 17
    w2 = w.copy()
    w2[lat.indices == 17] = np.inf
    st, p, _ = dg.sssp(cuda(w2), 3, 17)
    assert st == _lib.ORSP_NO_PATH
    # path longer than path_cap -> overflow error, not a fault
    with pytest.raises(_lib.OrspError):
        dg.sssp(wt, 0, lat.N - 1, path_cap=3)
    # bad delta rejected on the host
    with pytest.raises(_lib.OrspError):
        dg.sssp(wt, 0, 1, delta=0.0)


def test_batch_bbox_matches_oracle():
    lat = build_lattice(90, 70, 6)
    w = uniform_weights(lat, seed=5, blocked_frac=0.03)
    dg = DeviceGraph.from_lattice(lat)
    boxes, src, dst = random_boxes(lat, 300, seed=9, lo=(2, 2, 1), hi=(90, 70, 6))
    # boxes larger than the shared-memory distance array (24K nodes) take the
    # global-memory path of the kernel
    rng = np.random.default_rng(1)
    big_boxes = np.array([[0, 89, 0, 69, 0, 5], [3, 85, 1, 66, 0, 5], [0, 89, 10, 69, 0, 5]] * 4, np.int32)
    bs = lat.node(rng.integers(3, 85, 12), rng.integers(10, 66, 12), rng.integers(0, 6, 12)).astype(np.int32)
    bd = lat.node(rng.integers(3, 85, 12), rng.integers(10, 66, 12), rng.integers(0, 6, 12)).astype(np.int32)
    boxes = np.concatenate([boxes, big_boxes])
    src = np.concatenate([src, bs])
    dst = np.concatenate([dst, bd])
    cap = 2048
    nodes, edges, lens = dg.batch_bbox(cuda(w), cuda(src), cuda(dst), cuda(boxes), path_cap=cap)
    ref_nodes, ref_lens = O.batch_bbox(lat.indptr, lat.indices, w, lat.nx, lat.ny, lat.nz, src, dst, boxes, cap)
    lens = lens.cpu().numpy()
    nodes = nodes.cpu().numpy()
    edges = edges.cpu().numpy()
    big = 0
    for k in range(len(src)):
        L = int(ref_lens[k])
        vol = (boxes[k, 1] - boxes[k, 0] + 1) * (boxes[k, 3] - boxes[k, 2] + 1) * (boxes[k, 5] - boxes[k, 4] + 1)
        big += vol > 24 * 1024
        if L < 2:
            assert lens[k] < 2, f"search {k}: oracle has no path"
            continue
        assert lens[k] == L, f"search {k}"
        assert np.array_equal(nodes[k, :L], ref_nodes[k, :L]), f"search {k}"
        assert np.array_equal(edges[k, : L - 1], O.path_to_edges(lat.indptr, lat.indices, ref_nodes[k, :L]))
    assert big > 0, "no box exercised the global-memory path"


def test_batch_bbox_empty_and_bad_box():
    lat = build_lattice(12, 12, 4)
    dg = DeviceGraph.from_lattice(lat)
    w = cuda(np.ones(lat.E, np.float32))
    z = torch.zeros(0, dtype=torch.int32, device="cuda")
    nodes, edges, lens = dg.batch_bbox(w, z, z, torch.zeros((0, 6), dtype=torch.int32, device="cuda"))
    assert lens.numel() == 0
    bad = cuda(np.array([[0, 20, 0, 3, 0, 3]], np.int32))
    with pytest.raises(_lib.OrspError):
        dg.batch_bbox(w, cuda(np.array([0], np.int32)), cuda(np.array([5], np.int32)), bad)


# ---------------------------------------------------------------- ROI, edges
def test_roi_bfs_matches_reference(golden):
    g = golden("golden_roi.npz")
    dg = DeviceGraph(g["indptr"], g["indices"])
    for k in range(int(g["ncases"])):
        s, d, depth, max_nodes = (int(v) for v in g[f"c{k}_args"])
        roi, g2r = dg.roi_bfs(s, d, min(depth, 150), max_nodes)
        roi = roi.cpu().numpy()
        assert np.array_equal(roi, g[f"c{k}_roi"]), f"case {k}"
        g2r = g2r.cpu().numpy()
        assert np.array_equal(g2r[roi], np.arange(len(roi)))
        assert (g2r >= 0).sum() == len(roi)


def test_path_to_edges_matches_reference(golden):
    g = golden("golden_path_edges.npz")
    d = golden("golden_dijkstra.npz")
    dg = DeviceGraph(d["ref_indptr"], d["ref_indices"])
    for k in range(int(g["n"])):
        e = dg.path_to_edges(cuda(g[f"p{k}"]))
        assert np.array_equal(e.cpu().numpy(), g[f"e{k}"])
