"""The oracle's snapshot-group schedule (CPU): groups of one net are the
plain per-net loop; repair rounds bring a group's first iteration back
towards the plain loop's overuse; and a net flagged for repair is the later
of two nets of a round that share an edge."""
import dataclasses

import numpy as np

from oracle.negotiate import route_plain
from orthoroute_b200.lattice import board_uniform_pins
from orthoroute_b200.negotiate import NegotiationConfig


def _cfg(**kw):
    base = dict(max_iterations=5, reroute="offenders", roi_margin=4, cost_update="net", full_graph_retry=False,
                net_order="disjoint")
    base.update(kw)
    return NegotiationConfig(**base)


def test_groups_of_one_are_the_plain_loop():
    b = board_uniform_pins(30, 26, 4, 40, seed=3)
    r0 = route_plain(b.lattice, b.src, b.dst, _cfg())
    r1 = route_plain(b.lattice, b.src, b.dst, _cfg(group_nets=1, group_repair=2))
    assert r0["trace"] == r1["trace"]
    assert all(np.array_equal(x, y) for x, y in zip(r0["paths"], r1["paths"]))
    assert np.array_equal(r0["usage"], r1["usage"])


def test_repair_rounds_reduce_first_iteration_overuse():
    b = board_uniform_pins(30, 26, 4, 60, seed=5)
    plain = route_plain(b.lattice, b.src, b.dst, dataclasses.replace(_cfg(), max_iterations=1))["trace"][0][0]
    snap = route_plain(b.lattice, b.src, b.dst, _cfg(group_nets=12, group_repair=0, max_iterations=1))["trace"][0][0]
    rep = route_plain(b.lattice, b.src, b.dst, _cfg(group_nets=12, group_repair=3, max_iterations=1))["trace"][0][0]
    assert rep <= snap and snap > plain
    assert rep <= plain + (snap - plain) // 2


def test_conflict_rule_flags_the_later_net():
    # the rule the device test kernel applies: owner[e] = the smallest rank
    # using e; net j is flagged when some e of its path has owner[e] < j
    paths = [np.array([1, 2, 3]), np.array([5, 6]), np.array([7, 3, 9]), np.array([6, 1])]
    owner = {}
    for j, p in enumerate(paths):
        for e in p.tolist():
            owner.setdefault(e, j)
    flags = [any(owner[e] < j for e in p.tolist()) for j, p in enumerate(paths)]
    assert flags == [False, False, True, True]
