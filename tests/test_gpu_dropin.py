"""The CUDA drop-in (orthoroute_b200.dropin) under the reference's own call
stream, and the ROI tile search it relies on.

The tape (tests/golden/golden_dropin_tape.npz) holds every call the
unmodified reference router made into the hot path while routing the
100x100x4 board with 200 nets for three iterations.  Replaying it through
the drop-in objects checks, call for call: every accountant update (each
array's bits after the call), every ROI, every search path (against the
fp32 oracle's answer recorded beside the reference's), every path -> edge
mapping and both via steps."""
import ctypes
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import oracle as O  # noqa: E402
from orthoroute_b200.tape import Tape, replay  # noqa: E402
from orthoroute_b200 import _lib  # noqa: E402
from orthoroute_b200.dropin import DropInROIExtractor, DropInSet, MirroredEdgeAccountant, install  # noqa: E402
from orthoroute_b200.lattice import build_lattice, uniform_weights  # noqa: E402
from orthoroute_b200.solver import DeviceGraph, GpuSolver  # noqa: E402

TAPE = Path(__file__).resolve().parent / "golden" / "golden_dropin_tape.npz"


@pytest.fixture(scope="module")
def tape():
    O.build_oracle()
    return Tape.load(TAPE)


def test_dropin_replays_the_reference_tape(tape):
    m = tape.meta
    lat = build_lattice(m["nx"], m["ny"], m["nz"])
    ds = DropInSet(lat.indptr, lat.indices, lattice=lat, nx=lat.nx, ny=lat.ny, nz=lat.nz)
    rep = replay(tape, ds, sync=torch.cuda.synchronize)
    assert not rep.failures, rep.failures[:5]
    assert rep.searches == sum(1 for ev in tape.events if ev["k"] == "search") > 300
    assert rep.paths_equal_oracle == rep.searches
    overs = [ev["out"] for ev in tape.events if ev["k"] == "acct" and ev["m"] == "compute_overuse"]
    assert [tuple(o) for o in overs[-len(m["trace"]):]] == [(s, c) for _, s, c in m["trace"]]
    # the cost array crossed to the device once per write, not once per search
    assert rep.calls["find_path_roi"] == rep.searches


def test_roi_node_list_searches_match_oracle():
    """orsp_sssp_roi_nodes (ROI tile sweeps on ROI-masked weights, ties by
    ROI index) against the oracle: BFS ROIs, ROIs with nodes appended out of
    order and repeated, fractional costs with exact ties, blocked edges, and
    src / dst outside the ROI."""
    rng = np.random.default_rng(31)
    for nx, ny, nz in ((60, 44, 4), (37, 53, 6), (90, 20, 3)):
        lat = build_lattice(nx, ny, nz)
        dg = DeviceGraph.from_lattice(lat)
        assert dg.is_lattice
        for case in range(24):
            w = uniform_weights(lat, seed=case, blocked_frac=float(rng.choice([0.0, 0.05, 0.2])))
            if case % 3 == 0:  # integer costs: many equal-distance ties
                w = np.where(np.isfinite(w), np.floor(w * 2), w).astype(np.float32)
            s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
            roi, _ = O.roi_bfs(lat.indptr, lat.indices, s, d, int(rng.integers(2, 60)),
                               int(rng.choice([50_000, 3000, 400])))
            roi = roi.astype(np.int32)
            if case % 4 == 1:  # must-keep style appends, a repeat (last index wins)
                extra = rng.choice(lat.N, size=5).astype(np.int32)
                roi = np.concatenate([roi, extra, roi[:1]])
            if case % 7 == 3:  # an endpoint outside the ROI
                roi = roi[roi != d]
            g2r = np.full(lat.N, -1, np.int32)
            g2r[roi] = np.arange(len(roi), dtype=np.int32)
            ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            wt = torch.from_numpy(w).cuda()
            st, path = dg.sssp_roi_nodes(wt, s, d, torch.from_numpy(roi).cuda())
            got = path.cpu().tolist() if st == _lib.ORSP_OK else None
            assert got == (ref.tolist() if len(ref) > 1 else None), (nx, ny, nz, case)
            # the same search through a global_to_roi map (orsp_sssp)
            st2, p2, _ = dg.sssp(wt, s, d, roi_map=torch.from_numpy(g2r).cuda())
            got2 = p2.cpu().tolist() if st2 == _lib.ORSP_OK else None
            assert got2 == got, (nx, ny, nz, case)


@pytest.mark.parametrize("impl", ["cta", "grid"])
def test_roi_node_list_off_lattice_matches_oracle(impl, monkeypatch):
    """orsp_sssp_roi_nodes on a graph that is not a tile lattice (the
    reference's own Lattice3D shape: inner-layer planar edges, full via
    stacks with duplicate via edges, no lattice geometry given): the one-CTA
    search (ROI-local distances through global_to_roi) and the grid search
    against the oracle, with repeated ROI nodes, ties and endpoints outside
    the ROI."""
    monkeypatch.setenv("ORSP_ROI_NODES_IMPL", impl)
    rng = np.random.default_rng(57)
    for nx, ny, nz in ((50, 40, 6), (31, 67, 4)):
        lat = build_lattice(nx, ny, nz, planar="inner", vias="full", duplicate_vias=True)
        dg = DeviceGraph(lat.indptr, lat.indices)
        assert not dg.is_lattice
        for case in range(16):
            w = uniform_weights(lat, seed=100 + case, blocked_frac=float(rng.choice([0.0, 0.1])))
            if case % 3 == 0:
                w = np.where(np.isfinite(w), np.floor(w * 2), w).astype(np.float32)
            s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
            roi, _ = O.roi_bfs(lat.indptr, lat.indices, s, d, int(rng.integers(2, 50)),
                               int(rng.choice([50_000, 2500, 300])))
            roi = roi.astype(np.int32)
            if case % 4 == 1:
                roi = np.concatenate([roi, rng.choice(lat.N, size=7).astype(np.int32), roi[:2]])
            if case % 5 == 2:
                roi = roi[roi != s]
            g2r = np.full(lat.N, -1, np.int32)
            g2r[roi] = np.arange(len(roi), dtype=np.int32)
            ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
            st, path = dg.sssp_roi_nodes(torch.from_numpy(w).cuda(), s, d, torch.from_numpy(roi).cuda())
            got = path.cpu().tolist() if st == _lib.ORSP_OK else None
            assert got == (ref.tolist() if len(ref) > 1 else None), (nx, ny, nz, case, st)


def test_roi_map_distances_bit_exact_and_generic_agrees(monkeypatch):
    """Distances of a ROI search (tile sweeps) are the oracle's bit for bit
    inside the ROI and +inf outside; the generic near-far search gives the
    same paths."""
    lat = build_lattice(70, 50, 6)
    w = uniform_weights(lat, seed=3, blocked_frac=0.05)
    wt = torch.from_numpy(w).cuda()
    dg = DeviceGraph.from_lattice(lat)
    rng = np.random.default_rng(4)
    for k in range(6):
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        roi, g2r = O.roi_bfs(lat.indptr, lat.indices, s, d, 30, 50_000)
        _, ref, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [s], roi_map=g2r)
        dist = torch.empty(lat.N, dtype=torch.float32, device="cuda")
        st, _, _ = dg.sssp(wt, s, -1, roi_map=torch.from_numpy(g2r).cuda(), dist_out=dist)
        assert st == _lib.ORSP_OK
        assert np.array_equal(dist.cpu().numpy().view(np.uint32), ref.view(np.uint32)), k
        st, p_tile, _ = dg.sssp(wt, s, d, roi_map=torch.from_numpy(g2r).cuda())
        monkeypatch.setenv("ORSP_SSSP_IMPL", "generic")
        st2, p_gen, _ = dg.sssp(wt, s, d, roi_map=torch.from_numpy(g2r).cuda())
        monkeypatch.delenv("ORSP_SSSP_IMPL")
        assert st == st2
        if st == _lib.ORSP_OK:
            assert p_tile.cpu().tolist() == p_gen.cpu().tolist(), k


def test_roi_bfs_keep_matches_oracle():
    """orsp_roi_bfs_keep (portal seeds as must-keep nodes) against the oracle,
    whose keep-list rule is pinned on the reference (test_oracle_reference)."""
    rng = np.random.default_rng(9)
    lat = build_lattice(45, 38, 4)
    dg = DeviceGraph.from_lattice(lat)
    for case in range(30):
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        keep = [int(v) for v in rng.choice(lat.N, size=int(rng.integers(1, 12)))] + [s, d]
        depth = int(rng.integers(1, 40))
        max_nodes = int(rng.choice([50_000, 900, 120, 6]))
        ref, _ = O.roi_bfs(lat.indptr, lat.indices, s, d, depth, max_nodes, keep=keep)
        got = dg.roi_bfs_keep(s, d, depth, max_nodes, keep).cpu().numpy()
        assert np.array_equal(got, ref), case


def _fake_router(lat, w):
    """The attributes install() reads from an initialised PathFinderRouter."""
    graph = SimpleNamespace(indptr=lat.indptr, indices=lat.indices, base_costs=lat.base_cost)
    lattice = SimpleNamespace(x_steps=lat.nx, y_steps=lat.ny, layers=lat.nz,
                              idx_to_coord=lambda n: tuple(int(c) for c in lat.coords(int(n))))
    old_acct = SimpleNamespace(E=lat.E, canonical={3: 1}, present=np.zeros(lat.E, np.float32),
                               present_ema=np.zeros(lat.E, np.float32), history=np.zeros(lat.E, np.float32),
                               capacity=np.ones(lat.E, np.float32), total_cost=w.copy())
    old_acct.present[3] = 1.0
    solver = SimpleNamespace(find_path_roi=None, find_path_multisource_multisink=None, plane_size=lat.nx * lat.ny)
    r = SimpleNamespace(graph=graph, lattice=lattice, solver=solver, accounting=old_acct,
                        roi_extractor=SimpleNamespace(max_roi_nodes=50_000), config=SimpleNamespace(),
                        _path_to_edges=None, _apply_via_pooling_penalties=lambda pf: None,
                        _block_via_edges_with_collisions=lambda: None)
    return r


def test_install_wires_every_hook():
    lat = build_lattice(40, 36, 4)
    w = uniform_weights(lat, seed=8, blocked_frac=0.02)
    r = _fake_router(lat, w)
    solver = install(r)
    assert isinstance(solver, GpuSolver)
    assert isinstance(r.accounting, MirroredEdgeAccountant)
    assert isinstance(r.roi_extractor, DropInROIExtractor)
    assert r.solver.find_path_roi == solver.find_path_roi
    assert not hasattr(r.solver, "gpu_solver")
    # the state moved over
    assert r.accounting.canonical == {3: 1} and float(r.accounting.present[3]) == 1.0
    assert np.array_equal(r.accounting.total_cost, w)
    # one net the way _route_all routes it (UPF:4614-4785)
    s, d = 5, lat.N - 7
    roi, g2r = r.roi_extractor.extract_roi(s, d, initial_radius=40, stagnation_bonus=0.0)
    (sx, sy, _), (dx, dy, _) = lat.coords(s), lat.coords(d)
    radius = max(60, int(0.75 * (abs(int(dx) - int(sx)) + abs(int(dy) - int(sy)))))
    ref_roi, _ = O.roi_bfs(lat.indptr, lat.indices, s, d, min(radius, 150), 50_000)
    assert np.array_equal(roi, ref_roi)
    costs = r.accounting.total_cost
    path = r.solver.find_path_roi(s, d, costs, roi, g2r)
    ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s], dst=d, roi_map=g2r)
    assert path == ref.tolist()
    edges = r._path_to_edges(path)
    assert edges == O.path_to_edges(lat.indptr, lat.indices, np.asarray(path, np.int32)).tolist()
    r.accounting.commit_path(edges)
    assert float(r.accounting.present[edges[0]]) == 1.0
    # a host write to the cost array reaches the next search (write counter)
    costs[edges] = np.float32(1e9)
    p2 = r.solver.find_path_roi(s, d, costs, roi, g2r)
    w2 = w.copy()
    w2[edges] = np.float32(1e9)
    ref2, *_ = O.dijkstra(lat.indptr, lat.indices, w2, [s], dst=d, roi_map=g2r)
    assert p2 == ref2.tolist() and p2 != path
