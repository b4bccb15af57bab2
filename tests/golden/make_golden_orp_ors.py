"""Golden files for the .ORP / .ORS formats and the headless board mapping,
produced by the reference's own code on a hand-made board.

    python tests/golden/make_golden_orp_ors.py [--ref <OrthoRoute tree>]  (default: $ORTHOROUTE_REFERENCE)

From the reference (orthoroute/infrastructure/serialization/orp_exporter.py,
ors_exporter.py, main.py and algorithms/manhattan/unified_pathfinder.py):

  golden_board.orp          export_board_to_orp(board_data dict)
  golden_board_2l.orp       the same for a 2-layer board
  golden_board_fp.orp       the same for a board of componentless footprints (pad escapes)
  golden_orp.json           {"board_data": the input dict,
                             "converted": convert_orp_to_board_data(import_board_from_orp(golden_board.orp)),
                             "mapping": grid and pad-to-pad tasks of UnifiedPathFinder.initialize_graph +
                                        _parse_requests (portals off) on the Board main.py builds,
                             "portals": PadEscapePlanner portals and escape stubs
                                        (precompute_all_pad_escapes) and the portal-to-portal tasks
                                        of _parse_requests (portals on); per board}
  golden_solution.ors       export_solution_to_ors(payload, metrics, metadata)
  golden_ors.json           {"inputs": payload / metrics / metadata,
                             "imported": import_solution_from_ors(golden_solution.ors),
                             "payload": convert_ors_to_geometry_payload(...) tracks and vias}
"""
from __future__ import annotations

import argparse
import json
import logging
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def board_data():
    """Pads of several kinds: component pads, pads without a component, a
    through-hole pad, a B.Cu pad, an unconnected pad; nets of 1, 2 and 3 pads,
    pads near a rounding tie of the grid (SHORT) and a net whose two pads
    share a grid point (SAME)."""
    names = ["F.Cu", "In1.Cu", "In2.Cu", "In3.Cu", "In4.Cu", "B.Cu"]
    pads = []

    def pad(comp, name, net, x, y, layers=("F.Cu",), drill=None):
        pads.append({"component": comp, "name": name, "net_name": net, "net_code": 0, "x": x, "y": y,
                     "width": 0.3, "height": 0.3, "drill": drill, "layers": list(layers), "type": "smd"})

    for i in range(6):
        pad("J1", str(i + 1), f"D{i}", 101.2 + 0.8 * i, 52.0)
        pad("U2", f"A{i + 1}", f"D{i}", 104.0 + 1.2 * i, 61.7 - 0.4 * i)
    pad("U2", "B1", "CLK", 108.3, 58.1)
    pad("J1", "7", "CLK", 99.9, 50.3, layers=names, drill=0.8)
    pad("", "", "CLK", 112.5, 55.55)
    pad("R3", "1", "VBUS", 110.0, 49.8, layers=("B.Cu",))
    pad("R3", "2", "VBUS", 103.0, 63.1)
    pad("", "", "ALONE", 106.0, 57.0)
    pad("U2", "B2", "", 107.0, 59.0)
    pad("TP1", "1", "SHORT", 105.01, 54.99)
    pad("TP2", "1", "SHORT", 105.05, 55.02)
    pad("TP3", "1", "SAME", 106.4, 56.4)
    pad("TP4", "1", "SAME", 106.45, 56.42)
    nets = {}
    for p in pads:
        if p["net_name"]:
            nets.setdefault(p["net_name"], {"name": p["net_name"], "code": 0, "pads": []})["pads"].append(p)
    return {"filename": "golden.kicad_pcb", "x_min": 95.0, "y_min": 45.0, "x_max": 120.0, "y_max": 70.0,
            "width": 25.0, "height": 25.0, "layers": len(names), "layer_names": names, "pads": pads, "nets": nets,
            "grid_resolution": 0.4, "clearance": 0.15, "track_width": 0.2, "via_diameter": 0.5, "via_drill": 0.25}


def board_data_two_layers():
    """A 2-layer board (both layers carry both directions in the reference),
    a component with two pads of the same name (the later one keeps the pad
    key), pads without a component, and a net whose first two pads are on
    B.Cu and F.Cu."""
    names = ["F.Cu", "B.Cu"]
    pads = []

    def pad(comp, name, net, x, y, layers=("F.Cu",), drill=None):
        pads.append({"component": comp, "name": name, "net_name": net, "net_code": 0, "x": x, "y": y,
                     "width": 0.3, "height": 0.3, "drill": drill, "layers": list(layers), "type": "smd"})

    pad("U1", "1", "A", 10.0, 10.0)
    pad("U1", "1", "B", 12.4, 10.8)      # same pad key as the first pad
    pad("U1", "2", "A", 18.2, 14.6, layers=("B.Cu",))
    pad("J2", "1", "B", 9.3, 16.1, layers=names, drill=0.9)
    pad("", "", "C", 11.11, 12.49)
    pad("", "", "C", 15.55, 12.51, layers=("B.Cu",))
    pad("J2", "2", "D", 14.0, 9.0, layers=("B.Cu",))
    pad("U1", "3", "D", 16.0, 17.0)
    nets = {}
    for p in pads:
        nets.setdefault(p["net_name"], {"name": p["net_name"], "code": 0, "pads": []})["pads"].append(p)
    return {"filename": "two_layers.kicad_pcb", "x_min": 5.0, "y_min": 5.0, "x_max": 25.0, "y_max": 22.0,
            "width": 20.0, "height": 17.0, "layers": 2, "layer_names": names, "pads": pads, "nets": nets,
            "grid_resolution": 0.4}


def board_data_footprints():
    """Pad escapes under pressure: two footprints of componentless pads (2 rows
    x 8 at one-cell pitch, so they enter the clearance set), nets joining
    them, one-pad nets placed in escape paths as obstacles, and a net with a
    pad off its grid column (dropped from escape planning)."""
    names = ["F.Cu", "In1.Cu", "In2.Cu", "B.Cu"]
    pads, nets = [], {}

    def pad(net, x, y):
        p = {"component": "", "name": "", "net_name": net, "net_code": 0, "x": round(x, 4), "y": round(y, 4),
             "width": 0.3, "height": 0.3, "drill": None, "layers": ["F.Cu"], "type": "smd"}
        pads.append(p)
        nets.setdefault(net, {"name": net, "code": 0, "pads": []})["pads"].append(p)

    for i in range(8):
        for r in range(2):
            k = 2 * i + r
            pad(f"N{k}", 20.0 + 0.4 * i, 20.0 + 0.4 * r)
    for i in range(8):
        for r in range(2):
            k = 2 * (7 - i) + (1 - r)
            pad(f"N{k}", 24.8 + 0.4 * i, 27.2 + 0.4 * r)
    for m, (x, y) in enumerate([(20.5, 21.6), (21.3, 19.0), (22.1, 22.0), (26.0, 26.5), (27.7, 28.9)]):
        pad(f"OBS{m}", x, y)
    pad("OFF", 22.25, 24.0)
    pad("OFF", 26.0, 24.4)
    return {"filename": "footprints.kicad_pcb", "x_min": 15.0, "y_min": 15.0, "x_max": 35.0, "y_max": 35.0,
            "width": 20.0, "height": 20.0, "layers": len(names), "layer_names": names, "pads": pads,
            "nets": nets, "grid_resolution": 0.4}


def reference_portals(bd, upf_mod, models):
    """Portals, escape stubs and portal-to-portal tasks of the reference's
    default (portal_enabled) headless set-up (main.py:432-456)."""
    board = _reference_board(bd, models)
    cfg = upf_mod.PathFinderConfig()
    cfg.portal_enabled = True
    pf = upf_mod.UnifiedPathFinder(config=cfg, use_gpu=False)
    pf.initialize_graph(board)
    board._gui_pads = bd.get("pads", [])
    tracks, _ = pf.precompute_all_pad_escapes(board)
    tasks = pf._parse_requests(board.nets)
    portals = [[pid, int(p.x_idx), int(p.y_idx), int(p.pad_layer), int(p.delta_steps), int(p.direction),
                float(p.pad_x), float(p.pad_y), int(p.entry_layer)] for pid, p in pf.portals.items()]
    return {"portals": portals, "escape_tracks": jsonable(tracks),
            "tasks": {k: [int(a), int(b)] for k, (a, b) in tasks.items()},
            "trivial": {k: int(v[0]) for k, v in pf.net_paths.items() if len(v) == 1}}


def _reference_board(bd, models):
    """The Board main.py's headless flow builds from board_data (main.py:355-422)."""
    Board, Net, Pad, Component, Coordinate = models
    board = Board(id="headless-board", name=bd.get("filename", "board"), layer_count=bd.get("layers", 2))
    board.nets = []
    comps = {}
    for c in bd.get("components", []):
        cid = c.get("reference", c.get("id", ""))
        if cid:
            comps[cid] = Component(id=cid, reference=cid, value=c.get("value", ""), footprint=c.get("footprint", ""),
                                   position=Coordinate(x=c.get("x", 0.0), y=c.get("y", 0.0)),
                                   angle=c.get("rotation", 0.0))
    n_pads = 0
    for net_id, info in bd.get("nets", {}).items():
        net = Net(id=net_id, name=info.get("name", net_id))
        net.pads = []
        for pr in info.get("pads", []):
            if not isinstance(pr, dict):
                continue
            pname = pr.get("name", pr.get("id", ""))
            cid = pr.get("component", "")
            p = Pad(id=pname or pr.get("id", f"pad_{n_pads}"), component_id=cid, net_id=net_id,
                    position=Coordinate(x=pr.get("x", 0.0), y=pr.get("y", 0.0)),
                    size=(pr.get("width", 0.2), pr.get("height", 0.2)), drill_size=pr.get("drill"),
                    layer=pr.get("layers", ["F.Cu"])[0] if pr.get("layers") else "F.Cu")
            net.pads.append(p)
            n_pads += 1
            if not cid:
                cid = "GENERIC_COMPONENT"
                p.component_id = cid
            if cid not in comps:
                comps[cid] = Component(id=cid, reference=cid, value="", footprint="",
                                       position=Coordinate(x=p.position.x, y=p.position.y), pads=[])
            comps[cid].pads.append(p)
        board.nets.append(net)
    board.components = list(comps.values())
    board._kicad_bounds = bd.get("bounds", None)
    board.layer_names = bd.get("layer_names", [])
    return board


def reference_mapping(bd, upf_mod, models):
    """Grid and tasks as main.py's headless flow builds them, with the portals
    off (pad-to-pad tasks)."""
    board = _reference_board(bd, models)
    cfg = upf_mod.PathFinderConfig()
    cfg.portal_enabled = False
    pf = upf_mod.UnifiedPathFinder(config=cfg, use_gpu=False)
    pf.initialize_graph(board)
    tasks = pf._parse_requests(board.nets)
    g = pf.lattice.geom
    return {"x_steps": int(g.x_steps), "y_steps": int(g.y_steps), "layers": int(pf.lattice.layers),
            "grid_min_x": float(g.grid_min_x), "grid_min_y": float(g.grid_min_y), "pitch": float(g.pitch),
            "layer_directions": list(g.layer_directions), "tasks": {k: [int(a), int(b)] for k, (a, b) in tasks.items()},
            "trivial": {k: int(v[0]) for k, v in pf.net_paths.items() if len(v) == 1}}


def ors_inputs():
    tracks = [
        {"net": "D0", "layer": "In1.Cu", "x1": 101.2, "y1": 52.0, "x2": 101.2, "y2": 55.6, "width": 0.24},
        {"net": "D0", "layer": "In2.Cu", "x1": 101.2, "y1": 55.6, "x2": 104.0, "y2": 55.6, "width": 0.24},
        {"net_id": "CLK", "layer": "In3.Cu", "start": (99.9, 50.3), "end": (108.3, 50.3), "width": 0.2},
        {"net_id": "VBUS", "layer": "In4.Cu", "start_x": 110.0, "start_y": 49.8, "end_x": 110.0, "end_y": 63.1},
        {"layer": "In1.Cu", "x1": 1.0, "y1": 2.0, "x2": 3.0, "y2": 2.0},
    ]
    vias = [
        {"net": "D0", "x": 101.2, "y": 52.0, "from_layer": "F.Cu", "to_layer": "In1.Cu", "diameter": 0.5,
         "drill": 0.25},
        {"net_id": "CLK", "position": (108.3, 50.3), "from_layer": "In3.Cu", "to_layer": "F.Cu", "size": 0.6,
         "drill": 0.3},
        {"net_id": "VBUS", "position": {"x": 110.0, "y": 63.1}, "from_layer": "In4.Cu", "to_layer": "B.Cu"},
        {"net": "ALONE"},
    ]
    metrics = [
        {"iteration": 1, "overuse": 12, "routed_nets": 7, "overflow": 30.5},
        {"iteration": 2, "overuse_count": 3, "nets_routed": 8, "overflow_cost": 4.0, "wirelength": 88.2,
         "vias": 9, "time": 0.25},
        {"iteration": 3, "overuse": 0, "routed": 8, "iteration_time": 0.5, "via_count": 10},
    ]
    metadata = {"orthoroute_version": "0.2.0", "total_time": 12.5, "iterations": 3, "converged": True,
                "barrel_conflicts": 0, "nets_routed": 8, "wirelength": 90.0, "via_count": 4, "track_count": 5,
                "overflow": 0, "board_name": "golden"}
    return tracks, vias, metrics, metadata


def jsonable(o):
    return json.loads(json.dumps(o))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ORTHOROUTE_REFERENCE"),
                    required=not os.environ.get("ORTHOROUTE_REFERENCE"),
                    help="OrthoRoute source tree (default: $ORTHOROUTE_REFERENCE)")
    args = ap.parse_args()
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.dont_write_bytecode = True
    sys.path.insert(0, args.ref)
    logging.disable(logging.CRITICAL)
    from orthoroute.infrastructure.serialization.orp_exporter import (convert_orp_to_board_data,
                                                                       export_board_to_orp, import_board_from_orp)
    from orthoroute.infrastructure.serialization.ors_exporter import (convert_ors_to_geometry_payload,
                                                                       export_solution_to_ors,
                                                                       import_solution_from_ors)
    import orthoroute.algorithms.manhattan.unified_pathfinder as upf
    from orthoroute.domain.models.board import Board, Component, Coordinate, Net, Pad

    bd = board_data()
    orp_path = HERE / "golden_board.orp"
    export_board_to_orp(json.loads(json.dumps(bd)), str(orp_path), compress=True)
    converted = convert_orp_to_board_data(import_board_from_orp(str(orp_path)))
    models = (Board, Net, Pad, Component, Coordinate)
    mapping = reference_mapping(converted, upf, models)
    bd2 = board_data_two_layers()
    orp2 = HERE / "golden_board_2l.orp"
    export_board_to_orp(json.loads(json.dumps(bd2)), str(orp2), compress=True)
    converted2 = convert_orp_to_board_data(import_board_from_orp(str(orp2)))
    mapping2 = reference_mapping(converted2, upf, models)
    bd3 = board_data_footprints()
    orp3 = HERE / "golden_board_fp.orp"
    export_board_to_orp(json.loads(json.dumps(bd3)), str(orp3), compress=True)
    converted3 = convert_orp_to_board_data(import_board_from_orp(str(orp3)))
    mapping3 = reference_mapping(converted3, upf, models)
    portals = {sfx: reference_portals(cv, upf, models)
               for sfx, cv in (("", converted), ("_2l", converted2), ("_fp", converted3))}
    (HERE / "golden_orp.json").write_text(json.dumps({"board_data": bd, "converted": jsonable(converted),
                                                      "mapping": mapping, "board_data_2l": bd2,
                                                      "converted_2l": jsonable(converted2),
                                                      "mapping_2l": mapping2, "board_data_fp": bd3,
                                                      "converted_fp": jsonable(converted3),
                                                      "mapping_fp": mapping3,
                                                      **{"portals" + k: v for k, v in portals.items()}}, indent=1))

    tracks, vias, metrics, metadata = ors_inputs()

    class Payload:
        pass

    pl = Payload()
    pl.tracks, pl.vias = tracks, vias
    ors_path = HERE / "golden_solution.ors"
    export_solution_to_ors(pl, metrics, metadata, str(ors_path), compress=True)
    geom, meta = import_solution_from_ors(str(ors_path))
    back = convert_ors_to_geometry_payload(geom)
    (HERE / "golden_ors.json").write_text(json.dumps({
        "inputs": {"tracks": jsonable(tracks), "vias": jsonable(vias), "metrics": metrics, "metadata": metadata},
        "imported": {"geometry": geom, "metadata": meta},
        "payload": {"tracks": jsonable(back.tracks), "vias": jsonable(back.vias)}}, indent=1))
    for m in (mapping, mapping2, mapping3):
        print(f"tasks {len(m['tasks'])}, trivial {len(m['trivial'])}, grid {m['x_steps']}x{m['y_steps']}x{m['layers']}")
    for k, v in portals.items():
        print(f"portals{k}: {len(v['portals'])} portals, {len(v['escape_tracks'])} escape tracks, {len(v['tasks'])} tasks")


if __name__ == "__main__":
    main()
