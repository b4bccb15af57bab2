"""Host side of the negotiation schedules (no GPU): the level schedule of
box searches, its cut into device groups, and the first-fit disjoint-round
order, against their defining properties and the oracle's own rounds."""
import numpy as np

from oracle.negotiate import _first_fit_rounds
from orthoroute_b200.lattice import bbox_with_margin, board_uniform_pins
from orthoroute_b200.negotiate import disjoint_order, level_groups, level_schedule


def _meet(a, b):
    return a[0] <= b[1] and b[0] <= a[1] and a[2] <= b[3] and b[2] <= a[3] and a[4] <= b[5] and b[4] <= a[5]


def _boxes(seed=3, n=120):
    b = board_uniform_pins(60, 50, 4, n, seed=seed)
    return bbox_with_margin(b.lattice, b.src, b.dst, np.full(n, 3, dtype=np.int64))


def test_level_schedule_levels_are_disjoint_and_ordered():
    boxes = _boxes()
    lv = level_schedule(boxes)
    M = len(boxes)
    for j in range(M):
        earlier = [i for i in range(j) if _meet(boxes[i], boxes[j])]
        assert lv[j] == (max(lv[i] for i in earlier) + 1 if earlier else 0)
    for L in range(int(lv.max()) + 1):
        sel = np.nonzero(lv == L)[0]
        assert not any(_meet(boxes[a], boxes[b]) for x, a in enumerate(sel) for b in sel[:x])


def test_level_groups_cut_levels_in_order():
    boxes = _boxes(seed=4)
    idx = np.arange(len(boxes))
    lv = level_schedule(boxes)
    order, ptr = level_groups(idx, lv, group_max=5)
    assert sorted(order.tolist()) == idx.tolist()
    assert ptr[0] == 0 and ptr[-1] == len(idx) and np.all(np.diff(ptr) > 0) and np.all(np.diff(ptr) <= 5)
    for q in range(len(ptr) - 1):
        g = order[ptr[q]:ptr[q + 1]]
        assert len(set(lv[g].tolist())) == 1  # one level per group
        assert np.all(np.diff(g) > 0)  # original order kept
    assert np.all(np.diff(lv[order]) >= 0)  # level after level


def test_disjoint_order_is_first_fit_rounds():
    boxes = _boxes(seed=5, n=150)
    idx = np.random.default_rng(0).permutation(len(boxes))
    got = disjoint_order(boxes, idx)
    assert np.array_equal(got, _first_fit_rounds(boxes, idx))
    # under that order the level schedule is the rounds: non-decreasing levels
    lv = level_schedule(boxes[got])
    assert np.all(np.diff(lv) >= 0)
    assert disjoint_order(boxes, idx[:0]).size == 0
