"""Column-via lattices (the reference's own Lattice3D graph: planar edges on
the inner layers, vias between any two layers of a column, every via edge
duplicated) on the tile sweeps with the per-column via pass, against the
oracle and against the reference's recorded paths.  fp32 distances and
paths must be identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as O  # noqa: E402
from orthoroute_b200 import _lib  # noqa: E402
from orthoroute_b200.lattice import build_lattice, uniform_weights  # noqa: E402
from orthoroute_b200.solver import DeviceGraph, GpuSolver  # noqa: E402


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


def _ref_lattice(nx, ny, nz):
    return build_lattice(nx, ny, nz, planar="inner", vias="full", duplicate_vias=True)


def _weights(lat, seed, blocked, integer):
    w = uniform_weights(lat, seed=seed, blocked_frac=blocked)
    if integer:  # many equal-distance ties
        w = np.where(np.isfinite(w), np.floor(w * 2), w).astype(np.float32)
    return w


def test_reference_golden_graph_is_a_column_via_lattice(golden):
    """The graph the reference's Lattice3D built (golden_dijkstra.npz), with its
    dimensions: recognised as a column-via lattice, and every recorded
    reference path reproduced by the tile search."""
    g = golden("golden_dijkstra.npz")
    nx, ny, nz = (int(v) for v in g["ref_dims"])
    dg = DeviceGraph(g["ref_indptr"], g["ref_indices"], nx, ny, nz)
    assert dg.lattice_kind == 2 and dg.route_loop_ok
    solver = GpuSolver(dg)
    roi = np.arange(dg.N, dtype=np.int32)
    for k in range(int(g["nref"])):
        s, d = (int(v) for v in g[f"ref{k}_st"])
        p = solver.find_path_roi_gpu(s, d, g["ref_cost"], roi, roi)
        assert (p or []) == g[f"ref{k}_path"].tolist(), k


@pytest.mark.parametrize("shape,blocked,integer", [((40, 30, 6), 0.05, False), ((33, 17, 12), 0.0, True),
                                                   ((24, 20, 18), 0.03, False), ((19, 26, 4), 0.1, True)])
def test_column_via_full_and_box_searches_bit_exact(shape, blocked, integer):
    """Full searches (distances bit for bit), paths to random targets, and box
    searches (distances and paths with the box's ROI), 4 to 18 layers
    (the 18-layer case takes the deep-tile instantiation)."""
    lat = _ref_lattice(*shape)
    w = _weights(lat, sum(shape), blocked, integer)
    dg = DeviceGraph.from_lattice(lat)
    assert dg.lattice_kind == 2
    wt = torch.from_numpy(w).cuda()
    rng = np.random.default_rng(3)
    nxy = lat.nx * lat.ny
    for s in rng.choice(lat.N, size=3, replace=False):
        s = int(s)
        _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s])
        dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
        st, _, _ = dg.sssp(wt, s, -1, dist_out=dist)
        assert st == _lib.ORSP_OK
        assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), s
        for d in rng.choice(lat.N, size=3, replace=False):
            ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=int(d))
            st, p, _ = dg.sssp(wt, s, int(d))
            got = p.cpu().tolist() if st == _lib.ORSP_OK else []
            assert got == (ref.tolist() if len(ref) > 1 else []), (s, int(d))
    nx, ny, nz = shape
    for b in [(0, nx - 1, 0, ny - 1, 0, nz - 1), (2, nx // 2, 1, ny - 2, 0, nz - 1), (1, nx - 3, 3, ny // 2, 1, nz - 2)]:
        x0, x1, y0, y1, z0, z1 = b
        g2r = np.full(lat.N, -1, np.int32)
        zz, yy, xx = np.meshgrid(np.arange(z0, z1 + 1), np.arange(y0, y1 + 1), np.arange(x0, x1 + 1), indexing="ij")
        inside = (zz * nxy + yy * lat.nx + xx).ravel()
        g2r[inside] = np.arange(inside.size, dtype=np.int32)
        for _ in range(3):
            s, d = (int(inside[rng.integers(inside.size)]) for _ in range(2))
            _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s], roi_map=g2r)
            dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
            st, _, _ = dg.sssp_box(wt, s, -1, b, dist_out=dist)
            assert st == _lib.ORSP_OK
            assert np.array_equal(_bits(dist.cpu().numpy()), _bits(ref_dist)), (b, s)
            ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            st, p, _ = dg.sssp_box(wt, s, d, b)
            got = p.cpu().tolist() if (st == _lib.ORSP_OK and p is not None) else []
            assert got == (ref.tolist() if len(ref) > 1 else []), (b, s, d)


def test_column_via_roi_node_list_searches_match_oracle_and_cta():
    """BFS-ROI searches as the reference issues them (node lists with appended
    and repeated nodes, endpoints outside the ROI): the tile search on the
    column-via lattice, the oracle, and the one-CTA search on the same graph
    without its dimensions agree."""
    rng = np.random.default_rng(41)
    for shape in ((50, 40, 6), (31, 47, 10)):
        lat = _ref_lattice(*shape)
        dg = DeviceGraph.from_lattice(lat)
        flat = DeviceGraph(lat.indptr, lat.indices)
        assert dg.lattice_kind == 2 and not flat.is_lattice
        for case in range(14):
            w = _weights(lat, 200 + case, float(rng.choice([0.0, 0.08])), case % 3 == 0)
            wt = torch.from_numpy(w).cuda()
            s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
            roi, _ = O.roi_bfs(lat.indptr, lat.indices, s, d, int(rng.integers(2, 40)),
                               int(rng.choice([50_000, 2000, 300])))
            roi = roi.astype(np.int32)
            if case % 4 == 1:
                roi = np.concatenate([roi, rng.choice(lat.N, size=6).astype(np.int32), roi[:2]])
            if case % 5 == 2:
                roi = roi[roi != d]
            g2r = np.full(lat.N, -1, np.int32)
            g2r[roi] = np.arange(len(roi), dtype=np.int32)
            ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            want = ref.tolist() if len(ref) > 1 else None
            rt = torch.from_numpy(roi).cuda()
            st, p = dg.sssp_roi_nodes(wt, s, d, rt)
            assert (p.cpu().tolist() if st == _lib.ORSP_OK else None) == want, (shape, case)
            st2, p2 = flat.sssp_roi_nodes(wt, s, d, rt)
            assert (p2.cpu().tolist() if st2 == _lib.ORSP_OK else None) == want, (shape, case)


def test_column_via_multi_target_and_sources():
    """Seeds with start costs and targets with portal costs (targets are
    sinks) inside BFS ROIs, and many sources in one launch: the oracle's
    winner and path, and every distance row bit for bit."""
    lat = _ref_lattice(36, 28, 8)
    w = _weights(lat, 77, 0.04, False)
    dg = DeviceGraph.from_lattice(lat)
    solver = GpuSolver(dg)
    rng = np.random.default_rng(8)
    for i in range(12):
        ns, nt = int(rng.integers(1, 4)), int(rng.integers(1, 5))
        nodes = rng.choice(lat.N, size=ns + nt, replace=False)
        seeds, targets = nodes[:ns], nodes[ns:]
        scost = (rng.integers(0, 4, size=ns) * 0.5).astype(np.float32)
        tcost = rng.integers(0, 4, size=nt) * 0.25
        roi, g2r = O.roi_bfs(lat.indptr, lat.indices, int(seeds[0]), int(targets[0]), 30, 50_000)
        ref, _, _, _ = O.dijkstra(lat.indptr, lat.indices, w, seeds, roi_map=g2r, seed_cost=scost,
                                  targets=targets, target_cost=tcost)
        got = solver.find_path_multisource_multisink(list(zip(seeds.tolist(), scost.tolist())),
                                                     list(zip(targets.tolist(), tcost.tolist())), w, roi, g2r)
        if len(ref) < 2:
            assert got is None
        else:
            assert got is not None and got[0] == ref.tolist(), i
    wt = torch.from_numpy(w).cuda()
    src = [int(v) for v in rng.choice(lat.N, size=5, replace=False)]
    dist = torch.full((len(src), lat.N), float("nan"), dtype=torch.float32, device="cuda")
    assert dg.sssp_sources(wt, src, dist, per_launch=3) == _lib.ORSP_OK
    got = dist.cpu().numpy()
    for i, s in enumerate(src):
        _, ref_dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s])
        assert np.array_equal(_bits(got[i]), _bits(ref_dist)), (i, s)


@pytest.mark.parametrize("plan", [None, [{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}],
                                  [{"max_nodes": 1 << 40, "impl": 1, "tile_w": 32}]])
def test_column_via_batched_boxes_match_oracle(plan):
    """Batched box searches on a column-via lattice: one CTA per search, the
    tile sweeps with a distance slice per box and the column via pass, and a
    tile-32 plan (which column vias send to the one-CTA kernel): every path
    and every edge list (a via step maps to the first CSR edge) equal the
    oracle's."""
    from orthoroute_b200.lattice import random_boxes

    lat = _ref_lattice(48, 36, 6)
    w = _weights(lat, 5, 0.03, False)
    dg = DeviceGraph.from_lattice(lat)
    dg.set_batch_plan(plan)
    boxes, src, dst = random_boxes(lat, 120, seed=9, lo=(2, 2, 1), hi=(48, 36, 6))
    cap = 2048
    nodes, edges, lens = dg.batch_bbox(torch.from_numpy(w).cuda(), torch.from_numpy(src).cuda(),
                                       torch.from_numpy(dst).cuda(), torch.from_numpy(boxes).cuda(), path_cap=cap)
    ref_nodes, ref_lens = O.batch_bbox(lat.indptr, lat.indices, w, lat.nx, lat.ny, lat.nz, src, dst, boxes, cap)
    lens, nodes, edges = lens.cpu().numpy(), nodes.cpu().numpy(), edges.cpu().numpy()
    for k in range(len(src)):
        L = int(ref_lens[k])
        if L < 2:
            assert lens[k] < 2, k
            continue
        assert lens[k] == L, k
        assert np.array_equal(nodes[k, :L], ref_nodes[k, :L]), k
        assert np.array_equal(edges[k, : L - 1], O.path_to_edges(lat.indptr, lat.indices, ref_nodes[k, :L])), k


@pytest.mark.parametrize("order", ["index", "disjoint"])
def test_column_via_negotiation_matches_oracle(order):
    """The negotiation loop with per-net live costs on a column-via lattice
    (the device routing loop, one net or one group of disjoint boxes per
    launch): batched and sequential runs equal the oracle loop per iteration,
    per net and in the final edge usage."""
    from oracle.negotiate import route_plain
    from orthoroute_b200.lattice import board_uniform_pins
    from orthoroute_b200.negotiate import NegotiationConfig, PathFinder

    b = board_uniform_pins(40, 34, 6, 60, seed=8)
    lat = _ref_lattice(40, 34, 6)
    cfg = NegotiationConfig(max_iterations=5, reroute="offenders", roi_margin=3, cost_update="net",
                            full_graph_retry=False, net_order=order)
    ref = route_plain(lat, b.src, b.dst, cfg)
    pf = PathFinder(lat, config=cfg)
    assert pf.dg.lattice_kind == 2 and pf.dg.route_loop_ok
    rb = pf.route(b.src, b.dst, mode="batched")
    rs = pf.route(b.src, b.dst, mode="sequential")
    tr_ref = [(s, c) for s, c, _ in ref["trace"]]
    assert rb.overuse_trace() == tr_ref and rs.overuse_trace() == tr_ref
    for k in range(len(b.src)):
        assert np.array_equal(rb.paths[k], ref["paths"][k]), k
        assert np.array_equal(rs.paths[k], ref["paths"][k]), k
    assert np.array_equal(rb.edge_usage, ref["usage"]) and np.array_equal(rs.edge_usage, ref["usage"])


def test_column_via_snapshot_groups_match_oracle():
    """Snapshot groups with repair rounds (orsp_route_nets_snapshot) on a
    column-via lattice: the device loop equals the oracle loop of the same
    schedule per iteration, per net and in the final edge usage."""
    from oracle.negotiate import route_plain
    from orthoroute_b200.lattice import board_uniform_pins
    from orthoroute_b200.negotiate import NegotiationConfig, PathFinder

    b = board_uniform_pins(40, 34, 6, 60, seed=8)
    lat = _ref_lattice(40, 34, 6)
    cfg = NegotiationConfig(max_iterations=5, reroute="offenders", roi_margin=3, cost_update="net",
                            full_graph_retry=False, net_order="disjoint", group_nets=12, group_repair=2)
    ref = route_plain(lat, b.src, b.dst, cfg)
    pf = PathFinder(lat, config=cfg)
    assert pf.dg.lattice_kind == 2 and pf.dg.route_loop_ok
    rb = pf.route(b.src, b.dst, mode="batched")
    assert rb.overuse_trace() == [(s, c) for s, c, _ in ref["trace"]]
    for k in range(len(b.src)):
        assert np.array_equal(rb.paths[k], ref["paths"][k]), k
    assert np.array_equal(rb.edge_usage, ref["usage"])
