"""Headless routing of an .ORP board into an .ORS solution on the GPU path.

    python -m orthoroute_b200.headless board.ORP [-o board.ORS] [--max-iterations 200]
                                       [--mode batched|plain] [--warm] [--pitch 0.4]
                                       [--no-portals] [--vias adjacent|full]

The steps are those of the reference's `main.py headless` (main.py:287-622):
read the board (orp.read_orp / orp_to_board_data), build the routing lattice
and the tasks (portal to portal, or pad to pad), route with negotiated
congestion, emit tracks and vias, write the solution (ors.write_ors).  The board -> problem mapping
follows the reference's router:

* routing area: the pads of nets with two or more pads, plus 3 mm
  (PathFinderRouter._calc_bounds, unified_pathfinder.py:2254-2306); the board
  outline plus 3 mm when no net has two pads;
* grid: origin and extent rounded to the pitch, `int(span / pitch) + 1`
  steps (KiCadGeometry, pathfinder/kicad_geometry.py:23-34); F.Cu vertical,
  then alternating horizontal / vertical (kicad_geometry.py:41-49);
* pads: snapped to the nearest grid point, clamped, on their layer (the index
  of their first layer name; F.Cu otherwise) under the reference's pad keys,
  later pads with the same key replacing earlier ones (_pad_key / _map_pads,
  unified_pathfinder.py:2308-2385);
* tasks: each net's first two pads (_parse_requests,
  unified_pathfinder.py:2600-2650), a net whose two pads share a grid point
  being a one-node route.

Routing uses this package's lattice (planar edges on the inner layers of a
board with more than two layers, vias between adjacent layers, base cost 1
per grid step and 3 per via) and negotiate.PathFinder.

Portals (the reference's headless default, main.py:432-456; `--no-portals`
routes pad to pad): every pad of a routable net escapes along its column to a
portal (escapes.plan_escapes).  A net whose two pads both have a portal keeps
the reference's portal-to-portal task (entry-layer nodes,
unified_pathfinder.py:2629-2641), and its search runs between the portals'
F.Cu nodes, the reference's only search seeds (_get_portal_seeds,
unified_pathfinder.py:2495-2513), so the path itself drops the via from the
end of the stub to a routing layer.  The escape stubs go in front of the
routed tracks, duplicates removed by the reference's geometric key
(emit_geometry, unified_pathfinder.py:5690-5722).
"""
from __future__ import annotations

import argparse
import json
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple

import numpy as np

from .lattice import Lattice, build_lattice, layer_directions
from .orp import default_layer_names, orp_to_board_data, read_orp

ROUTING_MARGIN = 3.0  # mm
DEFAULT_PITCH = 0.4  # mm, the reference router's grid pitch


@dataclass
class HeadlessProblem:
    lattice: Lattice
    names: List[str]  # nets with a task, board order
    src: np.ndarray  # int32 node ids
    dst: np.ndarray
    trivial: Dict[str, int]  # nets whose two pads share a grid point -> that node
    grid_min_x: float
    grid_min_y: float
    pitch: float
    layer_names: List[str]
    layer_dirs: List[str]
    pad_nodes: Dict[str, int] = field(default_factory=dict)  # pad key -> grid node, the reference's order
    components: List[Tuple[str, List[Tuple[dict, str]]]] = field(default_factory=list)  # (component, [(pad, key)])
    net_pads: Dict[str, Tuple[str, str]] = field(default_factory=dict)  # net -> keys of its first two pads
    portals: Dict[str, object] = field(default_factory=dict)  # pad key -> escapes.Portal (portal runs)
    escape_tracks: List[dict] = field(default_factory=list)
    # search endpoints per task: src / dst, or the F.Cu nodes of both portals
    search_src: np.ndarray = None
    search_dst: np.ndarray = None
    vias: str = "full"  # the lattice's via set: "full" (the reference's) or "adjacent"


def routing_bounds(board_data: dict) -> Tuple[float, float, float, float]:
    xs, ys = [], []
    for net in board_data.get("nets", {}).values():
        pads = net.get("pads", [])
        if len(pads) >= 2:
            xs += [p.get("x", 0.0) for p in pads]
            ys += [p.get("y", 0.0) for p in pads]
    if xs:
        return (min(xs) - ROUTING_MARGIN, min(ys) - ROUTING_MARGIN, max(xs) + ROUTING_MARGIN,
                max(ys) + ROUTING_MARGIN)
    b = board_data.get("bounds")
    if b:
        return (b[0] - ROUTING_MARGIN, b[1] - ROUTING_MARGIN, b[2] + ROUTING_MARGIN, b[3] + ROUTING_MARGIN)
    return (0.0, 0.0, 100.0, 100.0)


def grid_geometry(bounds, pitch: float):
    """(grid_min_x, grid_min_y, x_steps, y_steps) with the reference's float
    arithmetic (Python round: half to even)."""
    min_x, min_y, max_x, max_y = bounds
    gx0, gy0 = round(min_x / pitch) * pitch, round(min_y / pitch) * pitch
    gx1, gy1 = round(max_x / pitch) * pitch, round(max_y / pitch) * pitch
    return gx0, gy0, int((gx1 - gx0) / pitch) + 1, int((gy1 - gy0) / pitch) + 1


def _pad_key(pad: dict, comp: str, pad_id: str) -> str:
    if comp == "GENERIC_COMPONENT":
        return f"{comp}_{pad_id}@{int(round(pad.get('x', 0.0) * 1000))},{int(round(pad.get('y', 0.0) * 1000))}"
    return f"{comp}_{pad_id}"


def build_problem(board_data: dict, pitch: float = DEFAULT_PITCH, portals: bool = False,
                  escape_seed: int = 42, vias: str = "full") -> HeadlessProblem:
    """The routing lattice and tasks of a board_data dict.  With portals, the
    pads escape to portals first (escapes.plan_escapes) and a net whose two
    pads both have one is routed between its portals, as the reference does
    with its default portal_enabled (unified_pathfinder.py:2629-2641).
    vias: "adjacent" (vias between neighbouring layers) or "full", the
    reference's via set (Lattice3D.get_legal_via_pairs, UPF:1136-1172: F.Cu
    to every routing layer and every pair of routing layers), searched as a
    column-via lattice."""
    nz = int(board_data.get("layers", 2))
    names = list(board_data.get("layer_names") or [])
    if len(names) < nz:
        names = default_layer_names(nz)
    gx0, gy0, nx, ny = grid_geometry(routing_bounds(board_data), pitch)
    lat = build_lattice(nx, ny, nz, planar="inner" if nz > 2 else "all", vias=vias)
    plane = nx * ny

    def snap(p) -> int:
        xi = min(max(round((p.get("x", 0.0) - gx0) / pitch), 0), nx - 1)
        yi = min(max(round((p.get("y", 0.0) - gy0) / pitch), 0), ny - 1)
        lay = (p.get("layers") or ["F.Cu"])[0]
        z = names.index(lay) if lay in names else 0
        return z * plane + yi * nx + xi

    # components in the order the reference's headless flow builds them: the
    # board's component list, then components first seen on net pads.  A
    # pad's id is its name, else its id, else pad_<k> with k the number of
    # pads built before it, nets in order (main.py:397-411).
    order: List[str] = []
    members: Dict[str, List[Tuple[dict, str]]] = {}
    for c in board_data.get("components", []):
        ref = c.get("reference", c.get("id", ""))
        if ref and ref not in members:
            members[ref] = []
            order.append(ref)
    net_pads: Dict[str, Tuple[str, str]] = {}
    k = 0
    for net_id, net in board_data.get("nets", {}).items():
        keys = []
        for p in net.get("pads", []):
            if not isinstance(p, dict):
                continue
            comp = p.get("component", "") or "GENERIC_COMPONENT"
            key = _pad_key(p, comp, p.get("name", p.get("id", "")) or p.get("id", f"pad_{k}"))
            k += 1
            keys.append(key)
            if comp not in members:
                members[comp] = []
                order.append(comp)
            members[comp].append((p, key))
        if len(keys) >= 2:
            net_pads[net_id] = (keys[0], keys[1])
    pad_nodes: Dict[str, int] = {}
    for comp in order:
        for p, key in members[comp]:
            pad_nodes[key] = snap(p)
    prob = HeadlessProblem(lat, [], np.zeros(0, np.int32), np.zeros(0, np.int32), {}, gx0, gy0, pitch, names,
                           layer_directions(nz), pad_nodes, [(c, members[c]) for c in order], net_pads)
    prob.vias = vias
    # a one-layer board has no routing layer to enter (the reference's
    # fallback there names layers 1 and 2, outside its lattice): pad to pad
    if portals and nz >= 2:
        from .escapes import plan_escapes
        prob.portals, prob.escape_tracks = plan_escapes(board_data, prob, seed=escape_seed)
    tnames, src, dst, ssrc, sdst, trivial = [], [], [], [], [], {}
    for net_id, (k1, k2) in net_pads.items():
        if k1 in prob.portals and k2 in prob.portals:
            a, b = prob.portals[k1], prob.portals[k2]
            s = a.entry_layer * plane + a.y_idx * nx + a.x_idx
            d = b.entry_layer * plane + b.y_idx * nx + b.x_idx
            s0, d0 = a.y_idx * nx + a.x_idx, b.y_idx * nx + b.x_idx
            if s0 == d0:  # both stubs end on one point: search between the entry-layer nodes
                s0, d0 = s, d
        else:
            s, d = pad_nodes[k1], pad_nodes[k2]
            s0, d0 = s, d
        if s != d:
            tnames.append(net_id)
            src.append(s)
            dst.append(d)
            ssrc.append(s0)
            sdst.append(d0)
        else:
            trivial[net_id] = s
    prob.names = tnames
    prob.src = np.asarray(src, np.int32)
    prob.dst = np.asarray(dst, np.int32)
    prob.search_src = np.asarray(ssrc, np.int32)
    prob.search_dst = np.asarray(sdst, np.int32)
    prob.trivial = trivial
    return prob


def portal_collisions(prob: HeadlessProblem) -> int:
    """Grid points where the portals of two or more pads of different nets
    end.  Their escape stubs meet there (a short in the planner's output).
    On this lattice a portal's F.Cu node has one via edge each way, so two
    searches that both leave (or both enter) the point share a directed edge
    and the route cannot reach zero overuse."""
    pad_net = {}
    for net, (k1, k2) in prob.net_pads.items():
        pad_net.setdefault(k1, net)
        pad_net.setdefault(k2, net)
    nets_at: Dict[Tuple[int, int], set] = {}
    for pid, pt in prob.portals.items():
        nets_at.setdefault((pt.x_idx, pt.y_idx), set()).add(pad_net.get(pid, pid))
    return sum(1 for v in nets_at.values() if len(v) > 1)


def forced_overuse(prob: HeadlessProblem) -> int:
    """A lower bound on the edges that stay overused: on a board of more than
    two layers an F.Cu node has no planar edges and one via edge each way, so
    every F.Cu search endpoint that several searches leave (or several enter)
    keeps that directed edge overused.  0 on boards of one or two layers."""
    if prob.lattice.nz <= 2 or prob.vias == "full":  # (full vias: an F.Cu node has one via to every layer)
        return 0
    plane = prob.lattice.nx * prob.lattice.ny
    out = 0
    for ends in (prob.search_src, prob.search_dst):
        vals, counts = np.unique(np.asarray(ends, np.int64), return_counts=True)
        out += int(np.sum((counts > 1) & (vals < plane)))
    return out


def merge_escapes(escape_tracks: List[dict], tracks: List[dict], vias: List[dict]):
    """Escape stubs in front of the routed tracks, later duplicates dropped
    by (net, layer, ends and width to 0.001 mm); vias deduplicated by (net,
    position, layers, drill, diameter) (unified_pathfinder.py:5690-5722)."""
    def dedupe(items, key):
        seen, out = set(), []
        for it in items:
            k = key(it)
            if k not in seen:
                seen.add(k)
                out.append(it)
        return out

    if not escape_tracks:
        return tracks, vias
    t = dedupe(list(escape_tracks) + list(tracks),
               lambda t: (t["net"], t["layer"], round(t["x1"], 3), round(t["y1"], 3), round(t["x2"], 3),
                          round(t["y2"], 3), round(t["width"], 3)))
    v = dedupe(list(vias), lambda v: (v["net"], round(v["x"], 3), round(v["y"], 3), v.get("from_layer"),
                                      v.get("to_layer"), round(v.get("drill", 0), 3), round(v.get("diameter", 0), 3)))
    return t, v


def headless_config(max_iterations: int = 200, groups: int = 0, repair: int = 3):
    """The negotiation schedule of headless runs: per-net live costs, only
    offending nets rerouted, bbox + 10-cell ROIs with a full-lattice retry,
    first-fit rounds of disjoint boxes; with groups > 0, batched runs take
    snapshot groups of that many nets with `repair` repair rounds."""
    from .negotiate import NegotiationConfig
    return NegotiationConfig(max_iterations=max_iterations, cost_update="net", reroute="offenders", roi_margin=10,
                             full_graph_retry=True, net_order="disjoint", group_nets=groups, group_repair=repair)


def route_board(board_data: dict, pitch: float = DEFAULT_PITCH, max_iterations: int = 200, mode: str = "batched",
                warm: bool = False, config=None, device=None, log=None, portals: bool = True,
                vias: str = "full", groups: int = 0):
    """Routes a board_data dict on the GPU (mode 'batched' or 'sequential'),
    through pad-escape portals unless portals is False, on a lattice with
    adjacent or full (the reference's) vias.  Returns (problem, RouteResult,
    tracks, vias, iteration metrics)."""
    from .geometry import generate_geometry
    from .negotiate import PathFinder

    prob = build_problem(board_data, pitch, portals=portals, vias=vias)
    cfg = config or headless_config(max_iterations, groups=groups)
    if vias == "full" and cfg.batch_plan is None:
        # the batched box searches on the tile sweeps (column vias)
        cfg.batch_plan = [{"max_nodes": 1 << 40, "impl": 1, "tile_w": 16}]
    pf = PathFinder(prob.lattice, config=cfg, device=device)
    hist = None
    if warm:
        from .warm import load_pretrained, warm_history_device
        net, scale = load_pretrained(device=pf.device)
        hist = warm_history_device(net, prob.lattice, prob.search_src, prob.search_dst, scale)
    metrics = []

    def cb(s):
        metrics.append({"iteration": s.iteration, "overuse": s.over_cnt, "overflow": s.over_sum,
                        "nets_routed": s.routed, "iteration_time": s.seconds})
        if log:
            log(f"iteration {s.iteration}: overuse {s.over_sum}/{s.over_cnt}, routed {s.routed}, {s.seconds:.2f} s")

    res = pf.route(prob.search_src, prob.search_dst, mode=mode, callback=cb, history_init=hist)
    net_paths = {}
    for name, path in zip(prob.names, res.paths):
        net_paths[name] = [int(v) for v in path] if path is not None and len(path) >= 2 else []
    for name, node in prob.trivial.items():
        net_paths[name] = [int(node)]
    tracks, vias = generate_geometry(pf.dg, net_paths, prob.layer_dirs, prob.grid_min_x, prob.grid_min_y, pitch,
                                     prob.layer_names, pitch)
    tracks, vias = merge_escapes(prob.escape_tracks, tracks, vias)
    return prob, res, tracks, vias, metrics


def run_headless(orp_file: str, output_file: Optional[str] = None, max_iterations: int = 200,
                 mode: str = "batched", warm: bool = False, pitch: float = DEFAULT_PITCH, log=print,
                 portals: bool = True, vias: str = "full", groups: int = 0) -> dict:
    """ORP in, ORS out; returns a summary of the run."""
    from .ors import GeometryPayload, write_ors

    t0 = time.perf_counter()
    board_data = orp_to_board_data(read_orp(orp_file))
    out = Path(output_file) if output_file else Path(orp_file).with_suffix(".ORS")
    via_style = vias
    prob, res, tracks, vias, metrics = route_board(board_data, pitch, max_iterations, mode, warm, log=log,
                                                   portals=portals, vias=via_style, groups=groups)
    total = time.perf_counter() - t0
    routed = sum(1 for p in res.paths if p is not None and len(p) >= 2) + len(prob.trivial)
    meta = {"orthoroute_version": "0.1.0", "board_name": board_data.get("filename", "board"), "total_time": total,
            "iterations": len(metrics), "total_iterations": len(metrics), "converged": bool(res.converged),
            "barrel_conflicts": 0, "nets_routed": routed, "wirelength": float(res.wirelength),
            "via_count": len(vias), "track_count": len(tracks),
            "overflow": metrics[-1]["overflow"] if metrics else 0}
    write_ors(GeometryPayload(tracks, vias), metrics, meta, out)
    summary = {"ors": str(out), "nets": len(prob.names) + len(prob.trivial), "routed": routed,
               "converged": bool(res.converged), "iterations": len(metrics), "tracks": len(tracks),
               "vias": len(vias), "seconds_total": round(total, 3), "seconds_route": round(res.seconds, 3),
               "lattice": [prob.lattice.nx, prob.lattice.ny, prob.lattice.nz], "lattice_vias": via_style,
               "snapshot_groups": groups, "searches": int(sum(s_.nets_searched for s_ in res.iterations)),
               "portals": len(prob.portals),
               "escape_tracks": len(prob.escape_tracks), "portal_collisions": portal_collisions(prob),
               "forced_overuse": forced_overuse(prob)}
    if log and summary["portal_collisions"]:
        log(f"warning: {summary['portal_collisions']} grid points hold the portals of two nets "
            "(their escape stubs meet, and the nets may share a via edge); --no-portals avoids them")
    if log:
        log(json.dumps(summary))
    return summary


def main(argv=None):
    ap = argparse.ArgumentParser(description="Route an .ORP board on the GPU and write an .ORS solution")
    ap.add_argument("orp")
    ap.add_argument("-o", "--output", default=None)
    ap.add_argument("--max-iterations", type=int, default=200)
    ap.add_argument("--mode", choices=["batched", "plain"], default="batched")
    ap.add_argument("--warm", action="store_true", help="start from the learned history prediction")
    ap.add_argument("--pitch", type=float, default=DEFAULT_PITCH)
    ap.add_argument("--no-portals", action="store_true", help="route pad to pad, without pad escapes")
    ap.add_argument("--vias", choices=["adjacent", "full"], default="full",
                    help="the reference's via set (F.Cu to every routing layer, every pair of routing layers; the "
                         "default), or vias between neighbouring layers only")
    ap.add_argument("--groups", type=int, default=0,
                    help="batched mode: snapshot groups of this many nets (one launch per group, then repair "
                         "rounds for nets sharing an edge); 0 keeps one launch per round of disjoint boxes")
    a = ap.parse_args(argv)
    s = run_headless(a.orp, a.output, a.max_iterations, "batched" if a.mode == "batched" else "sequential", a.warm,
                     a.pitch, portals=not a.no_portals, vias=a.vias, groups=a.groups)
    return 0 if s["converged"] else 1


if __name__ == "__main__":
    raise SystemExit(main())
