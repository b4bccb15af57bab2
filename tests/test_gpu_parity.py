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


def _lattice_env(monkeypatch, impl):
    """Selects the search implementation: generic near-far, or the tile sweeps
    with tile width 16/32 and the asynchronous, warp-specialised or round
    schedule, with plain or tensor-load (TMA) staging of whole-lattice tiles."""
    monkeypatch.setenv("ORSP_SSSP_IMPL", "generic" if impl == "generic" else "auto")
    monkeypatch.setenv("ORSP_LAT_TILE", "32" if impl == "lattice32" else "16")
    monkeypatch.setenv("ORSP_LAT_ASYNC", "0" if impl.endswith("rounds") else "1")
    monkeypatch.setenv("ORSP_LAT_SPEC", "1" if impl.endswith("spec") else "0")
    monkeypatch.setenv("ORSP_LAT_TMA", "1" if impl.endswith("tma") else "0")


@pytest.mark.parametrize("impl", ["lattice16", "lattice32", "lattice16-rounds", "lattice16-spec", "lattice16-tma",
                                  "generic"])
@pytest.mark.parametrize("shape,blocked,planar", [((60, 50, 6), 0.05, "all"), ((33, 17, 12), 0.0, "all"),
                                                  ((128, 96, 4), 0.03, "all"), ((45, 70, 6), 0.02, "inner")])
def test_sssp_full_distances_bit_exact(shape, blocked, planar, impl, monkeypatch):
    """Full searches, both implementations (tile sweeps on the lattice, generic
    near-far), both tile sizes and every schedule, bit-identical to the oracle."""
    _lattice_env(monkeypatch, impl)
    lat = build_lattice(*shape, planar=planar)
    w = uniform_weights(lat, seed=sum(shape), blocked_frac=blocked)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    rng = np.random.default_rng(7)
    for s in rng.choice(lat.N, size=3, replace=False):
        _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(s)])
        for delta in (0.37, 2.0, 1e4, 0.0):  # 0.0: width chosen on the device
            dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
            st, _, rounds = dg.sssp(wt, int(s), -1, delta=delta, dist_out=dist)
            assert st == _lib.ORSP_OK
            assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), f"src {s} delta {delta}"


@pytest.mark.parametrize("impl", ["lattice16", "lattice32", "lattice16-tma", "lattice16-spec", "generic"])
@pytest.mark.parametrize("shape,blocked,per_launch", [((60, 50, 6), 0.05, 0), ((33, 17, 12), 0.0, 3),
                                                      ((128, 96, 4), 0.03, 2), ((64, 40, 12), 0.02, 4)])
def test_sssp_sources_distances_bit_exact(shape, blocked, per_launch, impl, monkeypatch):
    """Many sources in one launch (whole-lattice boxes with their own
    distance rows, orsp_sssp_sources), in chunks of per_launch, a repeated
    source included: every row bit-identical to the oracle's full search, and
    a cost generation declared for the whole call."""
    _lattice_env(monkeypatch, impl)
    lat = build_lattice(*shape)
    w = uniform_weights(lat, seed=3 * sum(shape), blocked_frac=blocked)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    rng = np.random.default_rng(17)
    src = [int(v) for v in rng.choice(lat.N, size=6, replace=False)]
    src.append(src[1])
    for gen in (None, 5):
        dist = torch.full((len(src), lat.N), float("nan"), dtype=torch.float32, device="cuda")
        assert dg.sssp_sources(wt, src, dist, per_launch=per_launch, cost_generation=gen) == _lib.ORSP_OK
        got = dist.cpu().numpy()
        for i, s in enumerate(src):
            _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s])
            assert np.array_equal(_bits(got[i]), _bits(ref_dist)), (i, s, gen)
    # a single search after the call gathers the weights again when undeclared
    w2 = w.copy()
    w2[::7] = np.float32(1.5)
    wt.copy_(cuda(w2))
    d1 = torch.empty(lat.N, dtype=torch.float32, device="cuda")
    assert dg.sssp(wt, src[0], -1, dist_out=d1)[0] == _lib.ORSP_OK
    _, ref2, _, _ = O.dijkstra(lat.indptr, lat.indices, w2, [src[0]])
    assert np.array_equal(_bits(d1.cpu().numpy()), _bits(ref2))


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
    # bad delta rejected on the host (0.0 means "chosen on the device")
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(_lib.OrspError):
            dg.sssp(wt, 0, 1, delta=bad)


BATCH_PLANS = {
    "default": None,
    "sweeps16": [{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}],
    "sweeps32": [{"max_nodes": 1 << 40, "impl": 1, "tile_w": 32}],
    "mixed": [{"max_nodes": 800, "impl": 0, "delta": 0.75, "ctas_per_sm": 1},
              {"max_nodes": 6000, "impl": 0, "delta": 4.0, "ctas_per_sm": 3},
              {"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}],
}


@pytest.mark.parametrize("plan", list(BATCH_PLANS))
def test_batch_bbox_matches_oracle(plan):
    """Batched box searches under every tuning plan (one CTA per search, tile
    sweeps with a distance slice per box, mixed by box size) equal the oracle:
    every path and every edge list."""
    lat = build_lattice(90, 70, 6)
    w = uniform_weights(lat, seed=5, blocked_frac=0.03)
    dg = DeviceGraph.from_lattice(lat)
    dg.set_batch_plan(BATCH_PLANS[plan])
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


# ---------------------------------------------------------------- via pooling
def test_via_kernels_match_reference(golden):
    import oracle as O2

    g = golden("golden_via.npz")
    d = golden("golden_dijkstra.npz")
    nx, ny, nz = (int(v) for v in g["via_dims"])
    segz = nz - 2
    dg = DeviceGraph(d["ref_indptr"], d["ref_indices"], nx, ny, nz)
    lib = _lib.load()
    st = int(torch.cuda.current_stream().cuda_stream)
    # usage from the committed paths
    paths = [g[f"vpath{i}"] for i in range(int(g["npaths"]))]
    cap = max(len(p) for p in paths)
    nodes = np.zeros((len(paths), cap), np.int32)
    lens = np.array([len(p) for p in paths], np.int32)
    for i, p in enumerate(paths):
        nodes[i, : len(p)] = p
    # device copies are bound to names so they stay alive across each call
    nodes_d, lens_d = cuda(nodes), cuda(lens)
    col = torch.zeros(nx * ny, dtype=torch.int32, device="cuda")
    seg = torch.zeros(nx * ny * segz, dtype=torch.int32, device="cuda")
    assert lib.orsp_via_usage(dg.handle, len(paths), _lib.ptr(nodes_d), _lib.ptr(lens_d), cap,
                              _lib.ptr(col), _lib.ptr(seg), st) == 0
    assert np.array_equal(col.cpu().numpy().reshape(nx, ny), g["col_use"])
    assert np.array_equal(seg.cpu().numpy().reshape(nx, ny, segz), g["seg_use"])
    col_pres_in, seg_prefix_in = cuda(g["col_pres"]), cuda(g["seg_prefix"])
    col_cap, seg_cap = cuda(g["col_cap"].astype(np.int32)), cuda(g["seg_cap"].astype(np.int32))
    # penalties (float32 and float64 layer bias)
    for tag in ("f32", "f64"):
        total = cuda(g["total0"].copy())
        bias = cuda(g[f"bias_{tag}"].astype(np.float64))
        assert lib.orsp_via_penalties(dg.handle, _lib.ptr(col_pres_in), _lib.ptr(seg_prefix_in), _lib.ptr(bias),
                                      1 if tag == "f64" else 0, 0.20, 1.0, 1.0, 2.25, _lib.ptr(total), st) == 0
        assert np.array_equal(_bits(total.cpu().numpy()), _bits(g[f"pen_{tag}"])), tag
    # hard block
    total = cuda(g["total0"].copy())
    assert lib.orsp_via_hard_block(dg.handle, _lib.ptr(col), _lib.ptr(col_cap), _lib.ptr(seg), _lib.ptr(seg_cap),
                                   _lib.ptr(total), st) == 0
    assert np.array_equal(_bits(total.cpu().numpy()), _bits(g["blocked"]))
    # present smoothing + prefix vs the oracle restatement
    cp_ref, sp_ref, pre_ref = O2.via_present(g["col_use"], g["col_cap"], g["col_pres"], g["seg_use"], g["seg_cap"],
                                             g["seg_pres"])
    col_pres = cuda(g["col_pres"].copy())
    seg_pres = cuda(g["seg_pres"].copy())
    prefix = torch.zeros_like(seg_pres)
    assert lib.orsp_via_present(nx * ny, segz, _lib.ptr(col), _lib.ptr(col_cap), _lib.ptr(col_pres), _lib.ptr(seg),
                                _lib.ptr(seg_cap), _lib.ptr(seg_pres), _lib.ptr(prefix), 0.6, 0.4, st) == 0
    assert np.array_equal(_bits(col_pres.cpu().numpy()), _bits(cp_ref))
    assert np.array_equal(_bits(seg_pres.cpu().numpy()), _bits(sp_ref))
    assert np.array_equal(_bits(prefix.cpu().numpy()), _bits(pre_ref))


# ------------------------------------------------------- multi-source / sink
def test_sssp_multi_matches_oracle():
    """Seeds with start costs, targets with portal costs (targets are sinks),
    inside BFS ROIs and on the whole graph: same winner and same path as the
    oracle restatement of find_path_multisource_multisink."""
    lat = build_lattice(50, 40, 6)
    w = uniform_weights(lat, seed=21, blocked_frac=0.03)
    solver = GpuSolver(DeviceGraph.from_lattice(lat))
    rng = np.random.default_rng(5)
    for i in range(24):
        ns, nt = int(rng.integers(1, 5)), int(rng.integers(1, 6))
        nodes = rng.choice(lat.N, size=ns + nt, replace=False)
        seeds, targets = nodes[:ns], nodes[ns:]
        scost = (rng.integers(0, 4, size=ns) * 0.5).astype(np.float32)
        tcost = rng.integers(0, 4, size=nt) * 0.25
        if i % 2:
            roi, g2r = O.roi_bfs(lat.indptr, lat.indices, int(seeds[0]), int(targets[0]), 40, 50_000)
        else:
            roi = np.arange(lat.N, dtype=np.int32)
            g2r = roi
        ref, _, _, best = O.dijkstra(lat.indptr, lat.indices, w, seeds, roi_map=g2r, seed_cost=scost,
                                     targets=targets, target_cost=tcost)
        got = solver.find_path_multisource_multisink(list(zip(seeds.tolist(), scost.tolist())),
                                                     list(zip(targets.tolist(), tcost.tolist())), w, roi, g2r)
        if len(ref) < 2:
            assert got is None
        else:
            assert got is not None and got[0] == ref.tolist(), f"case {i}"
    # whole graph, allowed bitmap
    allowed = np.ones((lat.N + 31) // 32, dtype=np.uint32)
    allowed[:] = 0xFFFFFFFF
    blocked_nodes = rng.choice(lat.N, size=lat.N // 10, replace=False)
    for v in blocked_nodes:
        allowed[v >> 5] &= ~np.uint32(1 << (v & 31))
    ok = np.ones(lat.N, bool)
    ok[blocked_nodes] = False
    g2r = np.where(ok, np.arange(lat.N), -1).astype(np.int32)
    seeds = np.array([v for v in rng.choice(lat.N, 20) if ok[v]][:3], np.int32)
    targets = np.array([v for v in rng.choice(lat.N, 20) if ok[v]][:4], np.int32)
    ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, seeds, roi_map=g2r, targets=targets)
    got = solver.find_path_fullgraph_gpu_seeds(w, seeds, targets, allowed_bitmap=allowed, use_bitmap=True)
    assert (got or []) == (ref.tolist() if len(ref) > 1 else [])


def test_find_paths_on_rois_local_csr_batch():
    """13-tuple ROI batch (ROI-local CSRs) in one launch, with and without the
    per-ROI bitmap, against the oracle on each local CSR."""
    from orthoroute_b200.lattice import build_lattice as bl

    rng = np.random.default_rng(17)
    lat = bl(40, 30, 4)
    w = uniform_weights(lat, seed=2, blocked_frac=0.02)
    solver = GpuSolver(DeviceGraph.from_lattice(lat))
    batch, refs = [], []
    for k in range(40):
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        roi, g2r = O.roi_bfs(lat.indptr, lat.indices, s, d, int(rng.integers(3, 30)), 50_000)
        # local CSR of the ROI-induced subgraph, in ROI-index order
        ip = [0]
        ix, wl = [], []
        for u in roi:
            for e in range(lat.indptr[u], lat.indptr[u + 1]):
                v = lat.indices[e]
                if g2r[v] >= 0:
                    ix.append(g2r[v])
                    wl.append(w[e])
            ip.append(len(ix))
        ip = np.asarray(ip, np.int32)
        ix = np.asarray(ix, np.int32)
        wl = np.asarray(wl, np.float32)
        n = len(roi)
        bm = np.full((n + 31) // 32, 0xFFFFFFFF, dtype=np.uint32)
        if k % 3 == 0:  # clear some bits (never the endpoints)
            for v in rng.choice(n, size=max(1, n // 8), replace=False):
                if v not in (g2r[s], g2r[d]):
                    bm[v >> 5] &= ~np.uint32(1 << (v & 31))
        wl_ref = wl.copy()
        ok = ((bm[ix >> 5] >> (ix & 31).astype(np.uint32)) & 1) == 1
        wl_ref[~ok] = np.inf
        ref, *_ = O.dijkstra(ip, ix, wl_ref, [int(g2r[s])], dst=int(g2r[d]))
        batch.append((int(g2r[s]), int(g2r[d]), ip, ix, wl, n, bm, 0, 0, 0, 0, 0, 0))
        refs.append(ref.tolist() if len(ref) > 1 else None)
    got = solver.find_paths_on_rois(batch, use_bitmap=True)
    assert got == refs


def test_lattice_walk_long_runs_path_caps_and_deep_fallback():
    """The warp walk of the lattice backtraces: a 200-node straight run (many
    rounds of 32 lanes), a 30-layer via stack, path_cap exactly the path
    length (accepted) and one less (an error, or an error status per search
    in a batch); lattices deeper than a shared-memory tile take the generic
    search and the host routing loop, with the oracle's results."""
    lat = build_lattice(200, 6, 4)
    w = lat.base_cost.astype(np.float32)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    s, d = int(lat.node(0, 2, 1)), int(lat.node(199, 2, 1))
    ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d)
    assert len(ref) == 200
    full = (0, 199, 0, 5, 0, 3)
    for cap in (200, 4096):
        st, p, _ = dg.sssp_box(wt, s, d, full, path_cap=cap)
        assert st == _lib.ORSP_OK and p.cpu().tolist() == ref.tolist()
        st, p, _ = dg.sssp(wt, s, d, path_cap=cap)
        assert st == _lib.ORSP_OK and p.cpu().tolist() == ref.tolist()
    with pytest.raises(_lib.OrspError):
        dg.sssp_box(wt, s, d, full, path_cap=199)
    dg.set_batch_plan([{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}])
    boxes = np.array([full, full], np.int32)
    for cap, ok in ((200, True), (199, False)):
        nodes, edges, lens = dg.batch_bbox(wt, cuda(np.array([s, d], np.int32)), cuda(np.array([d, s], np.int32)),
                                           cuda(boxes), path_cap=cap)
        lens = lens.cpu().numpy()
        if ok:
            assert lens.tolist() == [200, 200]
            assert nodes.cpu().numpy()[0, :200].tolist() == ref.tolist()
        else:
            assert (lens < 0).all()

    stack = build_lattice(6, 6, 30)
    ws = stack.base_cost.astype(np.float32)
    dgs = DeviceGraph.from_lattice(stack)
    s, d = int(stack.node(3, 3, 0)), int(stack.node(3, 3, 29))
    ref, *_ = O.dijkstra(stack.indptr, stack.indices, ws, [s], dst=d)
    st, p, _ = dgs.sssp(cuda(ws), s, d)
    assert st == _lib.ORSP_OK and p.cpu().tolist() == ref.tolist() and len(ref) == 30

    deep = build_lattice(12, 10, 40)
    wd = uniform_weights(deep, seed=2, blocked_frac=0.02)
    dgd = DeviceGraph.from_lattice(deep)
    assert dgd.is_lattice and not dgd.route_loop_ok
    s = int(deep.node(1, 1, 0))
    _, ref_dist, _, _ = O.dijkstra(deep.indptr, deep.indices, wd, [s])
    dist = torch.empty(deep.N, dtype=torch.float32, device="cuda")
    st, _, _ = dgd.sssp(cuda(wd), s, -1, dist_out=dist)
    assert st == _lib.ORSP_OK and np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist))
    for b in [(0, 11, 0, 9, 0, 39), (2, 10, 1, 8, 5, 25)]:
        x0, x1, y0, y1, z0, z1 = b
        g2r = np.full(deep.N, -1, np.int32)
        zz, yy, xx = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1),
                                 indexing="ij")
        inside = deep.node(xx, yy, zz).ravel()
        g2r[inside] = np.arange(inside.size, dtype=np.int32)
        s, d = int(inside[3]), int(inside[-5])
        refp, *_ = O.dijkstra(deep.indptr, deep.indices, wd, [s], dst=d, roi_map=g2r)
        st, p, _ = dgd.sssp_box(cuda(wd), s, d, b)
        assert st == _lib.ORSP_OK and p.cpu().tolist() == refp.tolist(), b


@pytest.mark.parametrize("impl", ["lattice16", "lattice16-rounds"])
@pytest.mark.parametrize("shape", [(40, 36, 18), (35, 29, 13)])
def test_deep_lattice_bit_exact(shape, impl, monkeypatch):
    """Lattices and boxes of more than 12 layers (the tile kernel's deep
    instantiation, with the column load in 18-layer blocks): full-search
    distances, box paths in boxes deeper and shallower than 12 layers, and
    batched box searches with a distance slice per box, all equal to the
    oracle."""
    _lattice_env(monkeypatch, impl)
    lat = build_lattice(*shape)
    w = uniform_weights(lat, seed=sum(shape), blocked_frac=0.04)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    rng = np.random.default_rng(3)
    for s in rng.choice(lat.N, size=2, replace=False):
        _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(s)])
        dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
        st, _, _ = dg.sssp(wt, int(s), -1, dist_out=dist)
        assert st == _lib.ORSP_OK
        assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), f"src {s}"
    nx, ny, nz = shape
    nxy = nx * ny
    for b in [(0, nx - 1, 0, ny - 1, 0, nz - 1), (3, nx - 5, 2, ny - 4, 0, nz - 1), (5, 30, 4, 20, 2, 9)]:
        x0, x1, y0, y1, z0, z1 = b
        g2r = np.full(lat.N, -1, np.int32)
        zz, yy, xx = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        inside = (zz * nxy + yy * nx + xx).ravel()
        g2r[inside] = np.arange(inside.size, dtype=np.int32)
        for _ in range(3):
            s, d = (int(inside[rng.integers(inside.size)]) for _ in range(2))
            refp, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            st, p, _ = dg.sssp_box(wt, s, d, b)
            got = p.cpu().tolist() if (st == _lib.ORSP_OK and p is not None) else []
            assert got == (refp.tolist() if len(refp) > 1 else []), f"box {b} {s}->{d}"
    dg.set_batch_plan([{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}])
    boxes, src, dst = random_boxes(lat, 40, seed=11, lo=(4, 4, 13), hi=(nx, ny, nz))
    cap = 1024
    nodes, edges, lens = dg.batch_bbox(wt, cuda(src), cuda(dst), cuda(boxes), path_cap=cap)
    ref_nodes, ref_lens = O.batch_bbox(lat.indptr, lat.indices, w, nx, ny, nz, src, dst, boxes, cap)
    lens, nodes, edges = lens.cpu().numpy(), nodes.cpu().numpy(), edges.cpu().numpy()
    for k in range(len(src)):
        L = int(ref_lens[k])
        if L < 2:
            assert lens[k] < 2, f"search {k}: oracle has no path"
            continue
        assert lens[k] == L and np.array_equal(nodes[k, :L], ref_nodes[k, :L]), f"search {k}"
        assert np.array_equal(edges[k, : L - 1], O.path_to_edges(lat.indptr, lat.indices, ref_nodes[k, :L]))


@pytest.mark.parametrize("impl", ["lattice16", "lattice32", "lattice16-rounds", "lattice16-spec", "generic"])
def test_sssp_box_matches_box_roi_and_oracle(impl, monkeypatch):
    """orsp_sssp_box == orsp_sssp with the box's ROI map == the oracle with that
    ROI: distances (full searches) and paths, for boxes at the border, thin
    boxes, single-layer boxes and endpoints outside the box."""
    _lattice_env(monkeypatch, impl)
    lat = build_lattice(75, 58, 6)
    w = uniform_weights(lat, seed=21, blocked_frac=0.04)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    rng = np.random.default_rng(13)
    nxy = lat.nx * lat.ny
    boxes = [(0, 74, 0, 57, 0, 5), (0, 20, 30, 57, 0, 5), (40, 74, 0, 15, 1, 4), (10, 11, 5, 50, 0, 5),
             (5, 60, 20, 20, 0, 5), (3, 40, 3, 40, 2, 2), (17, 49, 9, 33, 0, 3)]
    for k, b in enumerate(boxes):
        x0, x1, y0, y1, z0, z1 = b
        g2r = np.full(lat.N, -1, np.int32)
        zz, yy, xx = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        inside = (zz * nxy + yy * lat.nx + xx).ravel()
        g2r[inside] = np.arange(inside.size, dtype=np.int32)
        for j in range(4):
            s = int(inside[rng.integers(inside.size)])
            d = int(inside[rng.integers(inside.size)]) if j < 3 else int(rng.integers(lat.N))
            ref, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=-1, roi_map=g2r)
            dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
            st, _, _ = dg.sssp_box(wt, s, -1, b, dist_out=dist)
            assert st == _lib.ORSP_OK
            assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), f"box {k} src {s}"
            refp, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            st, p, _ = dg.sssp_box(wt, s, d, b)
            got = p.cpu().tolist() if (st == _lib.ORSP_OK and p is not None) else []
            assert got == (refp.tolist() if len(refp) > 1 else []), f"box {k} {s}->{d}"
            st2, p2, _ = dg.sssp(wt, s, d, roi_map=cuda(g2r))
            got2 = p2.cpu().tolist() if (st2 == _lib.ORSP_OK and p2 is not None) else []
            assert got2 == got
    # a source outside the box reaches nothing
    st, p, _ = dg.sssp_box(wt, 0, 5, (10, 20, 10, 20, 0, 5))
    assert st == _lib.ORSP_NO_PATH
    for bad in [(0, 75, 0, 10, 0, 5), (5, 4, 0, 10, 0, 5), (0, 10, -1, 10, 0, 5), (0, 10, 0, 10, 0, 6)]:
        with pytest.raises(_lib.OrspError):
            dg.sssp_box(wt, 0, 5, bad)


def test_batch_plans_agree_on_status_codes():
    """The per-search status of batch_bbox is the same under both
    implementations: source outside its box (-1), unreachable target (0),
    src == dst (one node), and ordinary paths."""
    lat = build_lattice(40, 30, 4)
    w = uniform_weights(lat, seed=3, blocked_frac=0.0)
    w2 = w.copy()
    w2[lat.indices == lat.node(20, 15, 2)] = np.inf  # node (20,15,2) cannot be entered
    dg = DeviceGraph.from_lattice(lat)
    boxes = np.array([[0, 9, 0, 9, 0, 3], [5, 30, 5, 25, 0, 3], [0, 39, 0, 29, 0, 3], [2, 12, 2, 12, 1, 2]],
                     np.int32)
    src = np.array([lat.node(20, 20, 0), lat.node(6, 6, 0), lat.node(1, 1, 3), lat.node(5, 5, 1)], np.int32)
    dst = np.array([lat.node(3, 3, 0), lat.node(20, 15, 2), lat.node(38, 28, 0), lat.node(5, 5, 1)], np.int32)
    out = {}
    for name in ("default", "sweeps16"):
        dg.set_batch_plan(BATCH_PLANS[name])
        nodes, edges, lens = dg.batch_bbox(cuda(w2), cuda(src), cuda(dst), cuda(boxes), path_cap=512)
        out[name] = (lens.cpu().numpy(), nodes.cpu().numpy())
    la, na = out["default"]
    lb, nb = out["sweeps16"]
    assert la.tolist() == lb.tolist()
    assert la[0] == -1 and la[1] == 0 and la[3] == 1 and la[2] >= 2
    assert np.array_equal(na[2, : la[2]], nb[2, : lb[2]])


@pytest.mark.parametrize("impl", ["lattice16", "lattice32", "lattice16-rounds", "lattice16-spec"])
def test_seed_on_tile_edge_single_layer_box(impl, monkeypatch):
    """A seed on a tile edge must reach the next tile even when no other cell
    of that edge improves: single-layer boxes (one routing axis), source on
    the first row or column of a tile, target in the neighbouring tile."""
    _lattice_env(monkeypatch, impl)
    lat = build_lattice(90, 70, 6)
    w = uniform_weights(lat, seed=5, blocked_frac=0.0)
    dg = DeviceGraph.from_lattice(lat)
    wt = cuda(w)
    tw = 32 if impl == "lattice32" else 16
    # V layer (z=2): y-runs; H layer (z=1): x-runs
    cases = [((62, 63, 50, 68, 2, 2), (62, 66, 2), (62, 51, 2)),
             ((10, 11, 3, 60, 2, 2), (10, 3 + 16, 2), (10, 4, 2)),
             ((5, 5 + tw + 8, 7, 8, 1, 1), (5 + tw, 7, 1), (6, 7, 1)),
             ((5, 5 + tw + 8, 7, 8, 1, 1), (5 + tw - 1, 8, 1), (5 + tw + 7, 8, 1))]
    nxy = lat.nx * lat.ny
    for box, s3, d3 in cases:
        s, d = int(lat.node(*s3)), int(lat.node(*d3))
        g2r = np.full(lat.N, -1, np.int32)
        x0, x1, y0, y1, z0, z1 = box
        zz, yy, xx = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        inside = (zz * nxy + yy * lat.nx + xx).ravel()
        g2r[inside] = np.arange(inside.size, dtype=np.int32)
        ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
        assert len(ref) > 1
        st, p, _ = dg.sssp_box(wt, s, d, box)
        assert st == _lib.ORSP_OK and p.cpu().tolist() == ref.tolist(), f"{box} {s3}->{d3}"
        dg.set_batch_plan([{"max_nodes": 1 << 40, "impl": 1, "tile_w": tw}])
        nodes, _, lens = dg.batch_bbox(wt, cuda(np.array([s], np.int32)), cuda(np.array([d], np.int32)),
                                       cuda(np.array([box], np.int32)), path_cap=512)
        L = int(lens[0])
        assert L == len(ref) and nodes[0, :L].cpu().tolist() == ref.tolist()


def test_cost_generation_reuses_gathered_weights_only_when_declared():
    """orsp_graph_cost_generation: a whole-lattice search with the same array
    and generation as the last whole gather reuses the gathered weights; a new
    generation, an undeclared search or a box / ROI search in between gathers
    again, so every search sees the current costs."""
    lat = build_lattice(64, 48, 6)
    w = uniform_weights(lat, seed=5, blocked_frac=0.05)
    dg = DeviceGraph.from_lattice(lat)
    wt = torch.from_numpy(w).cuda()
    dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(2)

    def check(src, cost_host, gen):
        st, _, _ = dg.sssp(wt, int(src), -1, dist_out=dist, cost_generation=gen)
        _, ref, _, _ = O.dijkstra(lat.indptr, lat.indices, cost_host, [int(src)])
        assert st == 0 and np.array_equal(_bits(dist.cpu().numpy()), _bits(ref)), (src, gen)

    s = rng.choice(lat.N, size=6, replace=False)
    check(s[0], w, 7)
    check(s[1], w, 7)          # reused
    w2 = w.copy()
    w2[::3] = np.float32(2.5)
    wt.copy_(torch.from_numpy(w2))
    check(s[2], w2, 8)         # new generation: gathered again
    dg.sssp_box(wt, int(s[3]), -1, (0, 20, 0, 20, 0, lat.nz - 1))
    check(s[3], w2, 8)         # a box search rewrote part of the weights
    w3 = w2.copy()
    w3[1::5] = np.float32(1.25)
    wt.copy_(torch.from_numpy(w3))
    check(s[4], w3, None)      # undeclared: always gathered
    check(s[5], w3, 9)
