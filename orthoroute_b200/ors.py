""".ORS solution files (OrthoRoute Solution: gzip-compressed JSON, format 1.0).

The document is the reference's (orthoroute/infrastructure/serialization/
ors_exporter.py, "ORS" below), field for field, so that KiCad-side tools that
import the reference's solutions import these:

* ``solution_to_ors`` / ``write_ors``  export_solution_to_ors (ORS:18-96) with
  _build_solution_metadata, _build_geometry_data, _build_iteration_metrics and
  _build_statistics (ORS:99-339);
* ``read_ors``                         import_solution_from_ors (ORS:342-401);
* ``ors_to_geometry_payload``          convert_ors_to_geometry_payload (ORS:404-453).

The statistics keep the reference's arithmetic exactly: total wirelength
sums only tracks given as 'start'/'end' pairs or 'start_x'.. keys (tracks in
the router's own x1/y1/x2/y2 form count as zero length there), and the routed
net count falls back to distinct 'net_id' values of the tracks.
"""
from __future__ import annotations

from pathlib import Path
from typing import Any, Dict, List, Tuple

from .orp import FORMAT_VERSION, _dump_json, _load_json, utc_timestamp

ORS_SECTIONS = ("metadata", "geometry", "iteration_metrics", "statistics")


class GeometryPayload:
    """Tracks and vias of a solution (the shape the reference's geometry
    payload has: .tracks and .vias lists of dicts)."""

    def __init__(self, tracks: List[dict], vias: List[dict]):
        self.tracks = tracks
        self.vias = vias


def _track_xy(t: dict) -> Tuple[float, float, float, float]:
    if "start" in t and "end" in t:
        (a, b), (c, d) = t["start"], t["end"]
        return a, b, c, d
    if "x1" in t and "y1" in t:
        return t.get("x1", 0.0), t.get("y1", 0.0), t.get("x2", 0.0), t.get("y2", 0.0)
    return t.get("start_x", 0.0), t.get("start_y", 0.0), t.get("end_x", 0.0), t.get("end_y", 0.0)


def _geometry_section(geometry) -> Dict[str, Any]:
    by_net: Dict[str, dict] = {}
    layer_usage: Dict[Any, int] = {}

    def entry(net):
        if net not in by_net:
            by_net[net] = {"net_id": net, "tracks": [], "vias": []}
        return by_net[net]

    for t in geometry.tracks:
        net = str(t.get("net_id") or t.get("net", "unknown"))
        x1, y1, x2, y2 = _track_xy(t)
        layer = t.get("layer", 0)
        entry(net)["tracks"].append({"layer": layer, "start": {"x": float(x1), "y": float(y1)},
                                     "end": {"x": float(x2), "y": float(y2)}, "width": float(t.get("width", 0.15))})
        layer_usage[layer] = layer_usage.get(layer, 0) + 1
    for v in geometry.vias:
        net = str(v.get("net_id") or v.get("net", "unknown"))
        if "position" in v:
            pos = v["position"]
            px, py = pos if isinstance(pos, (list, tuple)) else (pos.get("x", 0.0), pos.get("y", 0.0))
        elif "x" in v and "y" in v:
            px, py = v.get("x", 0.0), v.get("y", 0.0)
        else:
            px, py = 0.0, 0.0
        entry(net)["vias"].append({"position": {"x": float(px), "y": float(py)},
                                   "from_layer": v.get("from_layer", 0), "to_layer": v.get("to_layer", 1),
                                   "diameter": float(v.get("size", 0.4)), "drill": float(v.get("drill", 0.2))})
    all_tracks, all_vias = [], []
    for d in by_net.values():
        all_tracks += [dict(t, net_id=d["net_id"]) for t in d["tracks"]]
        all_vias += [dict(v, net_id=d["net_id"]) for v in d["vias"]]
    return {"by_net": by_net, "all_tracks": all_tracks, "all_vias": all_vias, "layer_usage": layer_usage}


def _metrics_section(metrics: List[Dict[str, Any]]) -> List[Dict[str, Any]]:
    return [{
        "iteration": m.get("iteration", 0),
        "overuse_count": m.get("overuse_count", m.get("overuse", 0)),
        "nets_routed": m.get("nets_routed", m.get("routed", 0)),
        "overflow_cost": m.get("overflow_cost", m.get("overflow", 0.0)),
        "wirelength": m.get("wirelength", 0.0),
        "via_count": m.get("via_count", m.get("vias", 0)),
        "iteration_time_seconds": m.get("iteration_time", m.get("time", 0.0)),
    } for m in metrics]


def _statistics_section(geometry, metrics, metadata) -> Dict[str, Any]:
    wl = 0.0
    for t in geometry.tracks:
        if "start" in t and "end" in t:
            (x1, y1), (x2, y2) = t["start"], t["end"]
        else:
            x1, y1 = t.get("start_x", 0.0), t.get("start_y", 0.0)
            x2, y2 = t.get("end_x", 0.0), t.get("end_y", 0.0)
        dx, dy = x2 - x1, y2 - y1
        wl += (dx * dx + dy * dy) ** 0.5
    nets_routed = metadata.get("nets_routed", 0)
    if nets_routed == 0:
        nets_routed = len({str(t.get("net_id")) for t in geometry.tracks if t.get("net_id")})
    final_over, final_overflow = 0, 0.0
    if metrics:
        last = metrics[-1]
        final_over = last.get("overuse_count", last.get("overuse", 0))
        final_overflow = last.get("overflow_cost", last.get("overflow", 0.0))
    return {
        "total_tracks": len(geometry.tracks),
        "total_vias": len(geometry.vias),
        "total_wirelength_mm": wl,
        "nets_routed": nets_routed,
        "final_overuse_count": final_over,
        "final_overflow_cost": final_overflow,
        "converged": metadata.get("converged", final_over == 0),
        "iterations_completed": len(metrics),
    }


def solution_to_ors(geometry, iteration_metrics: List[Dict[str, Any]], metadata: Dict[str, Any],
                    timestamp: str = None) -> Dict[str, Any]:
    """The ORS document.  geometry: an object with .tracks and .vias (dicts
    as the router emits them); ValueError if it is None or lacks them."""
    if geometry is None:
        raise ValueError("Geometry cannot be None")
    if not hasattr(geometry, "tracks") or not hasattr(geometry, "vias"):
        raise ValueError("Geometry must have 'tracks' and 'vias' attributes")
    return {
        "format_version": FORMAT_VERSION,
        "metadata": {
            "export_timestamp": timestamp or utc_timestamp(),
            "orthoroute_version": metadata.get("orthoroute_version", "0.1.0"),
            "board_name": metadata.get("board_name", "unknown"),
            "total_iterations": metadata.get("total_iterations", 0),
            "converged": metadata.get("converged", False),
            "total_time_seconds": metadata.get("total_time", 0.0),
            "notes": metadata.get("notes", ""),
        },
        "geometry": _geometry_section(geometry),
        "iteration_metrics": _metrics_section(iteration_metrics),
        "statistics": _statistics_section(geometry, iteration_metrics, metadata),
    }


def write_ors(geometry, iteration_metrics, metadata, path, compress: bool = True) -> Dict[str, Any]:
    """Writes the solution as an .ORS file; returns the document written."""
    doc = solution_to_ors(geometry, iteration_metrics, metadata)
    _dump_json(doc, Path(path), compress)
    return doc


def read_ors(path) -> Tuple[Dict[str, Any], Dict[str, Any]]:
    """(geometry section, {'metadata', 'statistics', 'iteration_metrics'}).
    FileNotFoundError / ValueError as the reference's importer."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"ORS file not found: {path}")
    data = _load_json(path)
    version = data.get("format_version")
    if not version:
        raise ValueError("Missing format_version in ORS file")
    if version != FORMAT_VERSION:
        raise ValueError(f"Unsupported ORS format version: {version}")
    missing = [s for s in ORS_SECTIONS if s not in data]
    if missing:
        raise ValueError(f"Missing required sections: {', '.join(missing)}")
    return data["geometry"], {"metadata": data["metadata"], "statistics": data["statistics"],
                              "iteration_metrics": data["iteration_metrics"]}


def ors_to_geometry_payload(geometry_data: Dict[str, Any]) -> GeometryPayload:
    """Tracks and vias back in the router's dict form (positions as tuples,
    via 'diameter' as 'size')."""
    tracks = [{"net_id": t.get("net_id"), "layer": t.get("layer"), "start": (t["start"]["x"], t["start"]["y"]),
               "end": (t["end"]["x"], t["end"]["y"]), "width": t.get("width")}
              for t in geometry_data.get("all_tracks", [])]
    vias = [{"net_id": v.get("net_id"), "position": (v["position"]["x"], v["position"]["y"]),
             "from_layer": v.get("from_layer"), "to_layer": v.get("to_layer"), "size": v.get("diameter"),
             "drill": v.get("drill")} for v in geometry_data.get("all_vias", [])]
    return GeometryPayload(tracks, vias)

