"""The negotiation loop on the GPU: batched and sequential execution give the
same routes, and both match the oracle loop bit for bit (per-iteration
overuse, final paths, final edge usage)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle.negotiate import route_plain  # noqa: E402
from orthoroute_b200.lattice import board_uniform_pins  # noqa: E402
from orthoroute_b200.negotiate import NegotiationConfig, PathFinder  # noqa: E402


@pytest.mark.parametrize("reroute", ["all", "offenders"])
def test_negotiation_batched_sequential_oracle(reroute):
    b = board_uniform_pins(40, 36, 4, 60, seed=4)
    cfg = NegotiationConfig(max_iterations=6, reroute=reroute, roi_margin=4)
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    pf = PathFinder(b.lattice, config=cfg)
    rb = pf.route(b.src, b.dst, mode="batched")
    rs = pf.route(b.src, b.dst, mode="sequential")
    tr_ref = [(s, c) for s, c, _ in ref["trace"]]
    assert rb.overuse_trace() == tr_ref
    assert rs.overuse_trace() == tr_ref
    for k in range(len(b.src)):
        assert np.array_equal(rb.paths[k], ref["paths"][k]), f"net {k} (batched)"
        assert np.array_equal(rs.paths[k], ref["paths"][k]), f"net {k} (sequential)"
    assert np.array_equal(rb.edge_usage, ref["usage"])
    assert np.array_equal(rs.edge_usage, ref["usage"])


@pytest.mark.parametrize("reroute,order,grow,first", [("all", "index", 0, "sequential"),
                                                      ("offenders", "index", 0, "sequential"),
                                                      ("offenders", "disjoint", 0, "sequential"),
                                                      ("offenders", "disjoint", 3, "sequential"),
                                                      ("offenders", "disjoint", 3, "independent")])
def test_negotiation_per_net_costs_levels_match_sequential_and_oracle(reroute, order, grow, first):
    """Per-net (live usage) costs: the level-batched run equals the one-search-
    per-net run and the oracle, per iteration and per net, also with the
    first-fit disjoint order and with box growth for stalled nets."""
    b = board_uniform_pins(48, 40, 4, 70, seed=8)
    cfg = NegotiationConfig(max_iterations=5 if grow == 0 else 8, reroute=reroute, roi_margin=3,
                            cost_update="net", full_graph_retry=False, net_order=order, stall_grow=grow,
                            stall_iterations=1 if grow else 2, first_pass=first,
                            batch_plan=[{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}] if first == "independent"
                            else None)
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    pf = PathFinder(b.lattice, config=cfg)
    rb = pf.route(b.src, b.dst, mode="batched")
    rs = pf.route(b.src, b.dst, mode="sequential")
    tr_ref = [(s, c) for s, c, _ in ref["trace"]]
    assert rb.overuse_trace() == tr_ref
    assert rs.overuse_trace() == tr_ref
    for k in range(len(b.src)):
        assert np.array_equal(rb.paths[k], ref["paths"][k]), f"net {k} (batched)"
        assert np.array_equal(rs.paths[k], ref["paths"][k]), f"net {k} (sequential)"
    assert np.array_equal(rb.edge_usage, ref["usage"])


@pytest.mark.parametrize("reroute", ["all", "offenders"])
def test_device_routing_loop_equals_host_loop_and_oracle(reroute):
    """orsp_route_nets (the whole per-net loop enqueued on the device) equals
    the host-driven loop and the oracle: overuse per iteration, every path,
    the final usage and the final live costs."""
    import dataclasses

    b = board_uniform_pins(56, 44, 6, 90, seed=12)
    cfg = NegotiationConfig(max_iterations=6, reroute=reroute, roi_margin=4, cost_update="net",
                            full_graph_retry=False)
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    pf = PathFinder(b.lattice, config=cfg)
    assert pf.dg.is_lattice
    rd = pf.route(b.src, b.dst, mode="sequential")
    cost_dev = pf.acc.total_cost.cpu().numpy()
    pf_h = PathFinder(b.lattice, config=dataclasses.replace(cfg, native_loop=False))
    rh = pf_h.route(b.src, b.dst, mode="sequential")
    cost_host = pf_h.acc.total_cost.cpu().numpy()
    tr_ref = [(s, c) for s, c, _ in ref["trace"]]
    assert rd.overuse_trace() == tr_ref
    assert rh.overuse_trace() == tr_ref
    for k in range(len(b.src)):
        assert np.array_equal(rd.paths[k], ref["paths"][k]), f"net {k} (device loop)"
        assert np.array_equal(rh.paths[k], ref["paths"][k]), f"net {k} (host loop)"
    assert np.array_equal(rd.edge_usage, ref["usage"])
    assert np.array_equal(rh.edge_usage, ref["usage"])
    assert np.array_equal(cost_dev.view(np.uint32), cost_host.view(np.uint32))


def test_route_nets_group_contract():
    """orsp_route_nets: overlapping boxes in one group, a repeated net and a
    group_ptr that does not end at K are rejected on the host; a source
    outside its box gives no path; level groups equal one-net-at-a-time
    routing, costs included."""
    from orthoroute_b200 import _lib
    from orthoroute_b200._lib import ptr
    from orthoroute_b200.accounting import DeviceEdgeAccountant
    from orthoroute_b200.lattice import bbox_with_margin
    from orthoroute_b200.negotiate import level_groups, level_schedule

    b = board_uniform_pins(64, 48, 4, 40, seed=21)
    lat = b.lattice
    pf = PathFinder(lat, config=NegotiationConfig(cost_update="net"))
    lib = _lib.load()
    M = len(b.src)
    boxes = np.ascontiguousarray(bbox_with_margin(lat, b.src, b.dst, 2))
    cap = 512

    def run(order, groups, boxes_=boxes):
        acc = DeviceEdgeAccountant(lat.E, device=pf.device)
        acc.total_cost = pf.base.clone()
        nodes = torch.zeros((M, cap), dtype=torch.int32, device=pf.device)
        edges = torch.full((M, cap), -1, dtype=torch.int32, device=pf.device)
        lens = torch.zeros(M, dtype=torch.int32, device=pf.device)
        order = np.ascontiguousarray(order, dtype=np.int32)
        gp = None if groups is None else np.ascontiguousarray(groups, dtype=np.int32)
        st = lib.orsp_route_nets(pf.dg.handle, M, ptr(np.ascontiguousarray(b.src, np.int32)), ptr(b.dst),
                                 ptr(np.ascontiguousarray(boxes_, np.int32)), int(order.size), ptr(order),
                                 0 if gp is None else int(gp.size - 1), ptr(gp), ptr(nodes), ptr(edges), cap,
                                 ptr(lens), ptr(acc.total_cost), ptr(pf.base), ptr(acc.usage), ptr(acc.present),
                                 ptr(acc.capacity), ptr(acc.history), 0.5, 1.0, 1.0, 1.0, 1, 0)
        torch.cuda.synchronize()
        return st, nodes.cpu().numpy(), lens.cpu().numpy(), acc.usage.cpu().numpy(), acc.total_cost.cpu().numpy()

    lv = level_schedule(boxes)
    order, groups = level_groups(np.arange(M), lv)
    assert groups.size - 1 < M  # some launch holds several nets
    st1, n1, l1, u1, c1 = run(np.arange(M), None)
    st2, n2, l2, u2, c2 = run(order, groups)
    assert st1 == 0 and st2 == 0
    assert np.array_equal(l1, l2) and np.array_equal(u1, u2)
    assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32))
    for k in range(M):
        assert np.array_equal(n1[k, : l1[k]], n2[k, : l2[k]])
    i, j = next((i, j) for i in range(M) for j in range(i) if
                boxes[i, 0] <= boxes[j, 1] and boxes[j, 0] <= boxes[i, 1] and
                boxes[i, 2] <= boxes[j, 3] and boxes[j, 2] <= boxes[i, 3])
    assert run([j, i], [0, 2])[0] == _lib.ORSP_ERR_ARG
    assert run([0, 0], None)[0] == _lib.ORSP_ERR_ARG
    assert run(np.arange(M), [0, M // 2])[0] == _lib.ORSP_ERR_ARG
    # net 0 gets a box that does not hold its source: no path for it
    bx = boxes.copy()
    sx, sy = int(b.src[0] % lat.nx), int((b.src[0] // lat.nx) % lat.ny)
    bx[0] = (0, 3, 0, 3, 0, lat.nz - 1) if (sx > 3 or sy > 3) else (60, 63, 44, 47, 0, lat.nz - 1)
    st3, _, l3, _, _ = run(np.arange(M), None, boxes_=bx)
    assert st3 == 0 and l3[0] == 0


def test_negotiation_on_lattice_deeper_than_a_tile():
    """A 40-layer lattice (deeper than one shared-memory tile): the routing
    loop runs on the host over box searches that take the generic kernel,
    with the oracle's trace and paths."""
    b = board_uniform_pins(14, 12, 40, 8, seed=6)
    cfg = NegotiationConfig(max_iterations=4, roi_margin=3, cost_update="net", reroute="offenders")
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    pf = PathFinder(b.lattice, config=cfg)
    assert not pf.dg.route_loop_ok
    r = pf.route(b.src, b.dst, mode="sequential")
    assert r.overuse_trace() == [(s, c) for s, c, _ in ref["trace"]]
    for k in range(len(b.src)):
        assert np.array_equal(r.paths[k], ref["paths"][k]), f"net {k}"


@pytest.mark.parametrize("G,R", [(8, 0), (8, 2), (32, 3)])
def test_snapshot_groups_match_oracle(G, R):
    """orsp_route_nets_snapshot (groups of G overlapping boxes searched on one
    cost snapshot, then R repair rounds, all enqueued on the device) equals
    the host loop of the same schedule (one batch launch per round) and the
    oracle: overuse per iteration, every path, the final usage and live
    costs, and the search count."""
    import dataclasses

    b = board_uniform_pins(56, 44, 6, 90, seed=12)
    cfg = NegotiationConfig(max_iterations=6, reroute="offenders", roi_margin=4, cost_update="net",
                            full_graph_retry=False, net_order="disjoint", group_nets=G, group_repair=R)
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    pf = PathFinder(b.lattice, config=cfg)
    assert pf.dg.route_loop_ok
    rd = pf.route(b.src, b.dst, mode="batched")
    cost_dev = pf.acc.total_cost.cpu().numpy()
    pf_h = PathFinder(b.lattice, config=dataclasses.replace(cfg, native_loop=False))
    rh = pf_h.route(b.src, b.dst, mode="batched")
    cost_host = pf_h.acc.total_cost.cpu().numpy()
    tr_ref = [(s, c) for s, c, _ in ref["trace"]]
    assert rd.overuse_trace() == tr_ref
    assert rh.overuse_trace() == tr_ref
    assert [s.nets_searched for s in rd.iterations] == [s.nets_searched for s in rh.iterations]
    for k in range(len(b.src)):
        assert np.array_equal(rd.paths[k], ref["paths"][k]), f"net {k} (device loop)"
        assert np.array_equal(rh.paths[k], ref["paths"][k]), f"net {k} (host loop)"
    assert np.array_equal(rd.edge_usage, ref["usage"])
    assert np.array_equal(cost_dev.view(np.uint32), cost_host.view(np.uint32))


def test_snapshot_group_of_one_is_the_plain_loop():
    """Snapshot groups of one net (with repair rounds, which then never flag
    a net) give the plain per-net loop's routes bit for bit."""
    import dataclasses

    b = board_uniform_pins(48, 40, 6, 70, seed=21)
    cfg = NegotiationConfig(max_iterations=5, reroute="offenders", roi_margin=4, cost_update="net",
                            full_graph_retry=False, net_order="disjoint")
    r0 = PathFinder(b.lattice, config=cfg).route(b.src, b.dst, mode="batched")
    r1 = PathFinder(b.lattice, config=dataclasses.replace(cfg, group_nets=1, group_repair=2)).route(
        b.src, b.dst, mode="batched")
    assert r0.overuse_trace() == r1.overuse_trace()
    assert [s.nets_searched for s in r0.iterations] == [s.nets_searched for s in r1.iterations]
    assert all(np.array_equal(x, y) for x, y in zip(r0.paths, r1.paths))
    assert np.array_equal(r0.edge_usage, r1.edge_usage)


def test_snapshot_groups_deep_boxes_full_vias():
    """Snapshot groups on an 18-layer board (the deep-tile kernel on the
    boxes' own distance slices) match the host loop of the schedule."""
    import dataclasses

    from orthoroute_b200.lattice import board_footprints

    b = board_footprints(120, 100, 18, 160, None, seed=4)
    cfg = NegotiationConfig(max_iterations=4, reroute="offenders", roi_margin=6, cost_update="net",
                            full_graph_retry=False, net_order="disjoint", group_nets=16, group_repair=2)
    pf = PathFinder(b.lattice, config=cfg)
    rd = pf.route(b.src, b.dst, mode="batched")
    rh = PathFinder(b.lattice, config=dataclasses.replace(cfg, native_loop=False)).route(b.src, b.dst,
                                                                                         mode="batched")
    assert rd.overuse_trace() == rh.overuse_trace()
    assert all(np.array_equal(x, y) for x, y in zip(rd.paths, rh.paths))
    assert np.array_equal(rd.edge_usage, rh.edge_usage)
