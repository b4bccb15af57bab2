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


@pytest.mark.parametrize("reroute", ["all", "offenders"])
def test_negotiation_per_net_costs_levels_match_sequential_and_oracle(reroute):
    """Per-net (live usage) costs: the level-batched run equals the one-search-
    per-net run and the oracle, per iteration and per net."""
    b = board_uniform_pins(48, 40, 4, 70, seed=8)
    cfg = NegotiationConfig(max_iterations=5, reroute=reroute, roi_margin=3, cost_update="net",
                            full_graph_retry=False)
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
