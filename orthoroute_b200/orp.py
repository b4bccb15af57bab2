""".ORP board files (OrthoRoute PCB: gzip-compressed JSON, format 1.0).

The format and its field rules are the reference's
(orthoroute/infrastructure/serialization/orp_exporter.py, "ORP" below), so
that files move both ways between the two programs:

* ``read_orp``           import_board_from_orp (ORP:543-589): gzip or plain
                          JSON, version and section checks, same errors;
* ``orp_to_board_data``  convert_orp_to_board_data (ORP:592-766): the flat
                          board_data dict the reference's headless flow routes;
* ``board_data_to_orp``  export_board_to_orp for board_data dicts
                          (ORP:39-91 with the is_dict branches of the section
                          builders, ORP:94-540); ``write_orp`` writes it;
* ``synthetic_board_data`` a board of this package (lattice + two-pin nets,
                          lattice.Board) as a board_data dict, pins placed at
                          the world positions of their grid cells, so that the
                          benchmark boards can be exported as .ORP files.
"""
from __future__ import annotations

import gzip
import json
from datetime import datetime, timezone
from pathlib import Path
from typing import Any, Dict, List, Optional, Sequence

FORMAT_VERSION = "1.0"
ORP_SECTIONS = ("metadata", "board", "pads", "nets", "layers", "drc_rules", "grid_parameters")


def utc_timestamp() -> str:
    """UTC time as the reference writes it (ISO format, no offset, 'Z')."""
    return datetime.now(timezone.utc).replace(tzinfo=None).isoformat() + "Z"


def default_layer_names(layer_count: int) -> List[str]:
    """F.Cu, In1.Cu .. In(n-2).Cu, B.Cu (two layers: F.Cu, B.Cu)."""
    if layer_count == 2:
        return ["F.Cu", "B.Cu"]
    return ["F.Cu"] + [f"In{i}.Cu" for i in range(1, layer_count - 1)] + ["B.Cu"]


def make_pad_id(component_ref: str, pad_name: str, index: int) -> str:
    """Pad id of the format (ORP:19-36): 'REF@name', 'REF@index' without a
    pad name, 'PAD00042' without a component."""
    if component_ref and pad_name:
        return f"{component_ref}@{pad_name}"
    if component_ref:
        return f"{component_ref}@{index}"
    return f"PAD{index:05d}"


def _load_json(path: Path) -> Dict[str, Any]:
    try:
        with gzip.open(path, "rt", encoding="utf-8") as f:
            return json.load(f)
    except (gzip.BadGzipFile, OSError):
        with open(path, "r", encoding="utf-8") as f:
            return json.load(f)


def _dump_json(data: Dict[str, Any], path: Path, compress: bool) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    # gzip level 6: a quarter of level 9's time for a file about 5 % larger
    opener = (lambda: gzip.open(path, "wt", encoding="utf-8", compresslevel=6)) if compress else (
        lambda: open(path, "w", encoding="utf-8"))
    text = json.dumps(data, indent=2, ensure_ascii=False)  # one write: the same text as json.dump
    with opener() as f:
        f.write(text)


def read_orp(path) -> Dict[str, Any]:
    """The parsed file.  FileNotFoundError if it is missing; ValueError for a
    missing or unsupported format_version or missing sections."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"ORP file not found: {path}")
    data = _load_json(path)
    version = data.get("format_version")
    if not version:
        raise ValueError("Missing format_version in ORP file")
    if version != FORMAT_VERSION:
        raise ValueError(f"Unsupported ORP format version: {version}")
    missing = [s for s in ORP_SECTIONS if s not in data]
    if missing:
        raise ValueError(f"Missing required sections: {', '.join(missing)}")
    return data


def orp_to_board_data(orp: Dict[str, Any]) -> Dict[str, Any]:
    """The board_data dict of an ORP document: bounds, layers, pads (drilled
    pads on every layer, others on F.Cu or B.Cu), nets with their pads (by
    net name), components derived from the pads, default DRC rules and the
    grid pitch."""
    meta = orp.get("metadata", {})
    board = orp.get("board", {})
    b = board.get("bounds", {})
    layer_count = board.get("layer_count", 2)
    x_min, y_min = b.get("x_min", 0.0), b.get("y_min", 0.0)
    x_max, y_max = b.get("x_max", 0.0), b.get("y_max", 0.0)
    layer_names = [layer.get("name", f"Layer{i}") for i, layer in enumerate(orp.get("layers", []))]
    if not layer_names:
        layer_names = default_layer_names(layer_count)

    pads = []
    for p in orp.get("pads", []):
        pos, size = p.get("position", {}), p.get("size", {})
        drill = p.get("drill_size")
        if drill and drill > 0:
            layers, kind = layer_names, "thru_hole"
        else:
            layers, kind = (["B.Cu"] if p.get("layer", "F.Cu") == "B.Cu" else ["F.Cu"]), "smd"
        pid = p.get("id", "")
        pads.append({
            "id": pid,
            "component": p.get("component_ref", ""),
            "name": pid.split("@")[-1] if "@" in pid else "",
            "net_name": p.get("net_name", ""),
            "net_code": 0,
            "x": pos.get("x", 0.0),
            "y": pos.get("y", 0.0),
            "width": size.get("width", 0.0),
            "height": size.get("height", 0.0),
            "drill": drill,
            "layers": layers,
            "type": kind,
        })

    # each net's pads in pad order (grouped once instead of a scan per net)
    by_net: Dict[str, List[Dict[str, Any]]] = {}
    for p in pads:
        by_net.setdefault(p["net_name"], []).append(p)
    nets = {}
    for n in orp.get("nets", []):
        name = n.get("name", "")
        nets[name] = {"name": name, "code": 0, "pads": list(by_net.get(name, ()))}

    drc = orp.get("drc_rules", {})
    rules = drc.get("default", {})
    components = {}
    for p in pads:
        ref = p["component"]
        if ref and ref not in components:
            components[ref] = {"reference": ref, "value": "", "footprint": "", "x": p["x"], "y": p["y"]}

    return {
        "filename": meta.get("board_name", "Unknown Board"),
        "x_min": x_min,
        "y_min": y_min,
        "x_max": x_max,
        "y_max": y_max,
        "width": b.get("width", x_max - x_min),
        "height": b.get("height", y_max - y_min),
        "layers": layer_count,
        "layer_names": layer_names,
        "pads": pads,
        "nets": nets,
        "components": list(components.values()),
        "clearance": rules.get("clearance", 0.2),
        "track_width": rules.get("track_width", 0.25),
        "via_diameter": rules.get("via_diameter", 0.6),
        "via_drill": rules.get("via_drill", 0.3),
        "grid_resolution": orp.get("grid_parameters", {}).get("grid_pitch", 0.4),
        "airwires": [],
        "bounds": (x_min, y_min, x_max, y_max),
        "tracks": [],
        "zones": [],
        "drc_rules": drc,
    }


def board_data_to_orp(board_data: Dict[str, Any], filename: str = "board.orp",
                      timestamp: Optional[str] = None) -> Dict[str, Any]:
    """The ORP document of a board_data dict (pads keyed 'x', 'y',
    'component', 'name', 'net_name', 'layers', ...; nets keyed by name)."""
    bd = board_data
    pads_in = bd.get("pads", [])
    pads, pad_ids = [], []
    for i, p in enumerate(pads_in):
        ref = p.get("component", "")
        pid = make_pad_id(ref, p.get("name", str(i)), i)
        pad_ids.append(pid)
        layers = p.get("layers", ["F.Cu"])
        pads.append({
            "id": pid,
            "component_id": ref,
            "component_ref": ref,
            "net_id": p.get("net_name", ""),
            "net_name": p.get("net_name", ""),
            "position": {"x": p.get("x", 0.0), "y": p.get("y", 0.0)},
            "size": {"width": p.get("width", 0.0), "height": p.get("height", 0.0)},
            "drill_size": p.get("drill"),
            "layer": layers[0] if layers else "F.Cu",
            "shape": "circle",
            "angle": 0.0,
        })

    by_net: Dict[Any, List[int]] = {}
    for i, p in enumerate(pads_in):
        by_net.setdefault(p.get("net_name"), []).append(i)
    nets = []
    for name, net in bd.get("nets", {}).items():
        members = [(i, pads_in[i]) for i in by_net.get(name, ())]
        terminals = []
        for i, p in members:
            layers = p.get("layers", ["F.Cu"])
            terminals.append({"pad_id": pad_ids[i], "position": {"x": p.get("x", 0.0), "y": p.get("y", 0.0)},
                              "layer": layers[0] if layers else "F.Cu"})
        xs = [p.get("x", 0.0) for _, p in members]
        ys = [p.get("y", 0.0) for _, p in members]
        bounds = ({"x_min": min(xs), "y_min": min(ys), "x_max": max(xs), "y_max": max(ys)} if xs else
                  {"x_min": 0.0, "y_min": 0.0, "x_max": 0.0, "y_max": 0.0})
        nets.append({"id": name, "name": net.get("name", name), "netclass": "Default", "pad_count": len(members),
                     "is_routable": len(members) >= 2, "terminals": terminals, "bounds": bounds})

    layer_count = bd.get("layers", 2)
    names = bd.get("layer_names", []) or default_layer_names(layer_count)
    layers = [{"name": n, "type": "signal", "stackup_position": i, "thickness": 0.035, "material": "copper",
               "is_routing_layer": True} for i, n in enumerate(names[:layer_count])]

    x_min, y_min = bd.get("x_min", 0.0), bd.get("y_min", 0.0)
    x_max, y_max = bd.get("x_max", bd.get("width", 0.0)), bd.get("y_max", bd.get("height", 0.0))
    return {
        "format_version": FORMAT_VERSION,
        "metadata": {
            "filename": Path(filename).name,
            "board_name": bd.get("filename", "unknown.kicad_pcb"),
            "board_id": bd.get("filename", "unknown"),
            "export_timestamp": timestamp or utc_timestamp(),
            "orthoroute_version": "0.1.0",
        },
        "board": {
            "bounds": {"x_min": x_min, "y_min": y_min, "x_max": x_max, "y_max": y_max,
                       "width": bd.get("width", 0.0), "height": bd.get("height", 0.0)},
            "layer_count": layer_count,
            "thickness": bd.get("thickness", 1.6),
        },
        "pads": pads,
        "nets": nets,
        "layers": layers,
        "drc_rules": {
            "default": {"track_width": bd.get("track_width", 0.25), "clearance": bd.get("clearance", 0.2),
                        "via_diameter": bd.get("via_diameter", 0.6), "via_drill": bd.get("via_drill", 0.3),
                        "netclass": "Default"},
            "netclasses": {},
            "min_values": {"track_width": bd.get("min_track_width", 0.1),
                           "clearance": bd.get("min_clearance", 0.1),
                           "via_diameter": bd.get("min_via_diameter", 0.2),
                           "via_drill": bd.get("min_via_drill", 0.1)},
        },
        "grid_parameters": {
            "grid_pitch": bd.get("grid_resolution", 0.4),
            "expansion_margin": bd.get("expansion_margin", 3.0),
            "coordinate_system": "PCB coordinates in millimeters, origin at board bounds minimum",
            "board_bounds_used": {"x_min": x_min, "y_min": y_min, "x_max": x_max, "y_max": y_max},
        },
    }


def write_orp(board_data: Dict[str, Any], path, compress: bool = True) -> Dict[str, Any]:
    """Writes board_data as an .ORP file; returns the document written."""
    path = Path(path)
    doc = board_data_to_orp(board_data, filename=path.name)
    _dump_json(doc, path, compress)
    return doc


def synthetic_board_data(board, pitch: float = 0.4, origin=(10.0, 10.0),
                         layer_names: Optional[Sequence[str]] = None, name: str = "synthetic") -> Dict[str, Any]:
    """board_data for a lattice.Board: net k gets pads 'N{k}@1' (source) and
    'N{k}@2' (target) of component 'N{k}', at origin + (x, y) * pitch of their
    grid cells, SMD pads on their cell's layer (F.Cu or B.Cu; inner-layer
    cells are not pad positions and raise ValueError).  The origin should be
    a multiple of the pitch, so that the pads sit on the reference's grid."""
    lat = board.lattice
    names = list(layer_names) if layer_names else default_layer_names(lat.nz)
    ox, oy = origin
    pads, nets = [], {}
    for k, net in enumerate(board.names):
        members = []
        for j, node in enumerate((int(board.src[k]), int(board.dst[k]))):
            x, y, z = (int(v) for v in lat.coords(node))
            if z not in (0, lat.nz - 1):
                raise ValueError(f"net {net}: pin on inner layer {z}")
            pad = {"id": f"{net}@{j + 1}", "component": str(net), "name": str(j + 1), "net_name": str(net),
                   "net_code": k + 1, "x": ox + x * pitch, "y": oy + y * pitch, "width": 0.6 * pitch,
                   "height": 0.6 * pitch, "drill": None, "layers": [names[z]], "type": "smd"}
            pads.append(pad)
            members.append(pad)
        nets[str(net)] = {"name": str(net), "code": k + 1, "pads": members}
    w, h = (lat.nx - 1) * pitch, (lat.ny - 1) * pitch
    return {"filename": name, "x_min": ox, "y_min": oy, "x_max": ox + w, "y_max": oy + h, "width": w,
            "height": h, "layers": lat.nz, "layer_names": names, "pads": pads, "nets": nets,
            "grid_resolution": pitch}
