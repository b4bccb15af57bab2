"""Pad escapes and portals for headless runs (host side).

A restatement of the reference's PadEscapePlanner
(orthoroute/algorithms/manhattan/pad_escape_planner.py, "PEP" below) as its
headless flow runs it (main.py:449-456): every pad of a routable net (the
first two pads of a net with two or more pads) escapes along its grid column
to a portal 3..12 steps away, where routing starts on a randomly chosen
routing layer.  The same draws from the same seeded generator, in the same
order, give the reference's portals and escape stubs:

* pads snapped to the grid, dropped when more than half a step off a grid
  column, sorted by (column, row, pad key)                    PEP:232-295
* per column: escape direction away from the nearer neighbour (checkerboard
  when alone), length random in 3..min(12, half the gap, board edge),
  pairwise shortening of overlapping escapes, then a random entry layer and
  the first clearance-clean length (shorter first, then the other way)
                                                               PEP:487-687
* clearance: portal and three points of the stub at least 0.15 mm outside
  every other pad of the clearance set, looked up in a 5 mm grid
                                                               PEP:689-958
* stub geometry: vertical from the pad, a 45-degree tail when the pad is off
  its grid column                                              PEP:960-1035

The planner's gap-filling portals are switched off in the reference
(PEP:333-334) and are not restated.

Reference quirks kept for parity: pads are never skipped as through-hole
(the board model's pads have no 'drill' attribute), every pad counts as an
F.Cu pad, and only pads without a component (whose keys carry their
coordinates) enter the clearance set.
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass
from typing import Dict, List, Tuple

PAD_CLEARANCE_MM = 0.15
MIN_STEPS, MAX_STEPS = 3, 12
SNAP_MAX_STEPS = 0.5
INDEX_CELL_MM = 5.0
CHECK_RADIUS_MM = 3.0


@dataclass
class Portal:
    x_idx: int
    y_idx: int
    pad_layer: int
    delta_steps: int
    direction: int
    pad_x: float
    pad_y: float
    entry_layer: int


def _clearance_set(board_data: dict, pad_keys) -> Dict[str, dict]:
    """Pads whose keys carry coordinates ('...@x_um,y_um'), matched to the
    board's pads by position: for each pad, the first key (in key order)
    within 0.01 mm on both axes.  The keys are bucketed in 0.01 mm cells, so
    each pad tests only the keys of the cells around it with the same
    comparison."""
    cells: Dict[Tuple[int, int], List[Tuple[int, str, float, float]]] = {}
    for order, pid in enumerate(pad_keys):
        if "@" not in pid:
            continue
        try:
            xu, yu = map(int, pid.split("@")[1].split(","))
        except ValueError:
            continue
        kx, ky = xu / 1000.0, yu / 1000.0
        cells.setdefault((math.floor(kx / 0.01), math.floor(ky / 0.01)), []).append((order, pid, kx, ky))
    geoms = {}
    for p in board_data.get("pads", []):
        x, y = p["x"], p["y"]
        cx, cy = math.floor(x / 0.01), math.floor(y / 0.01)
        best = None
        for dx in (-2, -1, 0, 1, 2):  # a key within 0.01 mm lies at most one cell away; two for rounding
            for dy in (-2, -1, 0, 1, 2):
                for order, pid, kx, ky in cells.get((cx + dx, cy + dy), ()):
                    if (best is None or order < best[0]) and abs(kx - x) < 0.01 and abs(ky - y) < 0.01:
                        best = (order, pid)
        if best is not None:
            geoms[best[1]] = {"x": x, "y": y, "width": p["width"], "height": p["height"]}
    return geoms


def _index(geoms: Dict[str, dict]) -> Dict[Tuple[int, int], List[str]]:
    idx: Dict[Tuple[int, int], List[str]] = {}
    for pid, g in geoms.items():
        idx.setdefault((int(g["x"] / INDEX_CELL_MM), int(g["y"] / INDEX_CELL_MM)), []).append(pid)
    return idx


def _clear(x: float, y: float, own: str, geoms, index) -> bool:
    r = int(CHECK_RADIUS_MM / INDEX_CELL_MM) + 1
    cx, cy = int(x / INDEX_CELL_MM), int(y / INDEX_CELL_MM)
    for dx in range(-r, r + 1):
        for dy in range(-r, r + 1):
            for pid in index.get((cx + dx, cy + dy), ()):
                g = geoms[pid]
                if abs(g["x"] - x) > CHECK_RADIUS_MM or abs(g["y"] - y) > CHECK_RADIUS_MM or pid == own:
                    continue
                # keepout edges with the reference's operation order (a point
                # exactly on an edge is inside)
                x0 = g["x"] - g["width"] / 2.0 - PAD_CLEARANCE_MM
                x1 = g["x"] + g["width"] / 2.0 + PAD_CLEARANCE_MM
                y0 = g["y"] - g["height"] / 2.0 - PAD_CLEARANCE_MM
                y1 = g["y"] + g["height"] / 2.0 + PAD_CLEARANCE_MM
                if x0 <= x <= x1 and y0 <= y <= y1:
                    return False
    return True


def plan_escapes(board_data: dict, prob, seed: int = 42, grid_pitch: float = None):
    """(portals {pad key: Portal} in creation order, escape track dicts) for a
    board_data dict and its headless.HeadlessProblem."""
    rng = random.Random(seed)
    pitch = prob.pitch
    gp = grid_pitch if grid_pitch is not None else pitch
    nx, ny, nz = prob.lattice.nx, prob.lattice.ny, prob.lattice.nz
    geoms = _clearance_set(board_data, prob.pad_nodes.keys())
    index = _index(geoms)
    routable = set()
    for k1, k2 in prob.net_pads.values():
        routable.add(k1)
        routable.add(k2)

    pad_list = []
    for comp, pads in prob.components:
        for p, pid in pads:
            if pid not in routable:
                continue
            px, py = p.get("x", 0.0), p.get("y", 0.0)
            xi = min(max(round((px - prob.grid_min_x) / pitch), 0), nx - 1)
            yi = min(max(round((py - prob.grid_min_y) / pitch), 0), ny - 1)
            if abs(px - (prob.grid_min_x + xi * pitch)) / gp > SNAP_MAX_STEPS:
                continue
            pad_list.append((pid, xi, yi, px, py))
    pad_list.sort(key=lambda t: (t[1], t[2], t[0]))
    columns: Dict[int, list] = {}
    for pid, xi, yi, px, py in pad_list:
        columns.setdefault(xi, []).append((pid, yi, px, py))

    portals: Dict[str, Portal] = {}
    layers = list(range(1, nz)) or [1, 2]
    for xi in sorted(columns):
        col = columns[xi]
        plan = []
        for i, (pid, yi, px, py) in enumerate(col):
            below = yi - col[i - 1][1] if i > 0 else None
            above = col[i + 1][1] - yi if i < len(col) - 1 else None
            if above is not None and below is not None:
                d = 1 if above > below else -1
            elif above is not None:
                d = 1
            elif below is not None:
                d = -1
            else:
                d = -1 if (xi + yi) % 2 == 0 else 1
            edge = ny - 1 - yi if d > 0 else yi
            if d > 0 and above is not None:
                room = above // 2
            elif d < 0 and below is not None:
                room = below // 2
            else:
                room = MAX_STEPS
            top = max(min(MAX_STEPS, room, edge), MIN_STEPS)
            plan.append([pid, yi, d, rng.randint(MIN_STEPS, top), px, py])
        # Pairwise shortening of overlapping escapes, pairs in (i, j) order.
        # Lengths stay within MIN_STEPS..MAX_STEPS and the column is sorted
        # by row, so pads more than 2 * MAX_STEPS + 1 rows apart never
        # overlap; only those pairs are skipped (they neither hit nor change
        # a length).
        n = len(plan)
        reach = 2 * MAX_STEPS + 1
        for it in range(100):
            hit = False
            for i in range(n):
                a = plan[i]
                ya0 = a[1]
                for j in range(i + 1, n):
                    b = plan[j]
                    if b[1] - ya0 > reach:
                        break
                    if a[2] > 0:
                        lo_a, hi_a = ya0, ya0 + a[3]
                    else:
                        lo_a, hi_a = ya0 - a[3], ya0
                    if b[2] > 0:
                        lo_b, hi_b = b[1], b[1] + b[3]
                    else:
                        lo_b, hi_b = b[1] - b[3], b[1]
                    if not (hi_a + 1 < lo_b or hi_b + 1 < lo_a):
                        hit = True
                        if it % 2 == 0:
                            if a[3] > MIN_STEPS:
                                a[3] = max(MIN_STEPS, a[3] - 2)
                        elif b[3] > MIN_STEPS:
                            b[3] = max(MIN_STEPS, b[3] - 2)
            if not hit:
                break
        for pid, yi, d, delta, px, py in plan:
            entry = rng.choice(layers)

            def attempt(dd, steps):
                yp = yi + dd * steps
                wx, wy = prob.grid_min_x + xi * pitch, prob.grid_min_y + yp * pitch
                if not _clear(wx, wy, pid, geoms, index):
                    return None
                for t in (0.25, 0.5, 0.75):
                    if not _clear(px + t * (wx - px), py + t * (wy - py), pid, geoms, index):
                        return None
                return Portal(xi, yp, 0, steps, dd, px, py, entry)

            portal = None
            for steps in range(delta, MIN_STEPS - 1, -1):
                portal = attempt(d, steps)
                if portal:
                    break
            if not portal:
                far = min(MAX_STEPS, ny - 1 - yi if -d > 0 else yi)
                for steps in range(MIN_STEPS, far + 1):
                    portal = attempt(-d, steps)
                    if portal:
                        break
            if portal:
                portals[pid] = portal

    pad_net = {}
    for net, (k1, k2) in prob.net_pads.items():
        pad_net[k1] = net
        pad_net[k2] = net
    tracks = []
    lname = prob.layer_names[0] if prob.layer_names else "L0"
    for pid, pt in portals.items():
        net = pad_net.get(pid, f"PAD_{pid}")
        wx, wy = prob.grid_min_x + pt.x_idx * pitch, prob.grid_min_y + pt.y_idx * pitch
        dx, dy = wx - pt.pad_x, wy - pt.pad_y
        w = gp * 0.6
        if abs(dx) > 0.01:
            dy45 = (1 if dy > 0 else -1) * abs(dx)
            dyv = dy - dy45
            mx, my = pt.pad_x, pt.pad_y + dyv
            if abs(dyv) > 0.01:
                tracks.append({"net": net, "layer": lname, "x1": pt.pad_x, "y1": pt.pad_y, "x2": mx, "y2": my,
                               "width": w, "escape": True})
            tracks.append({"net": net, "layer": lname, "x1": mx, "y1": my, "x2": wx, "y2": wy, "width": w,
                           "escape": True})
        else:
            tracks.append({"net": net, "layer": lname, "x1": pt.pad_x, "y1": pt.pad_y, "x2": wx, "y2": wy,
                           "width": w, "escape": True})
    return portals, tracks
