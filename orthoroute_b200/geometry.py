"""Geometry emission: committed paths -> tracks and vias.

``generate_geometry`` returns what PathFinderRouter._generate_geometry_from_paths
(orthoroute/algorithms/manhattan/unified_pathfinder.py:5749-5834) returns -
track dicts {net, layer, x1, y1, x2, y2, width} and via dicts {net, x, y,
from_layer, to_layer, diameter, drill}, nets in dict order, each net's items
in emission order - with the path walk on the GPU (orsp_emit_geometry) and
the world mapping of _segment_world / _via_world (UPF:5596-5675) on the host:
lattice index -> grid_min + index * pitch, re-quantised to the grid.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .bookkeeping import _pack
from .solver import DeviceGraph, _stream


def _quantize(v, origin, pitch):
    return origin + np.round((v - origin) / pitch) * pitch


def generate_geometry(dg: DeviceGraph, net_paths: Dict[str, Sequence[int]], layer_dirs: Sequence[str],
                      grid_min_x: float, grid_min_y: float, pitch: float, layer_names: Sequence[str],
                      grid_pitch: float) -> Tuple[List[dict], List[dict]]:
    """layer_dirs: 'h' / 'v' / 'hv' per layer (Lattice3D.get_legal_axis);
    grid_pitch: the router's grid pitch (track width 0.6 * grid_pitch)."""
    items = [(n, p) for n, p in net_paths.items() if p is not None and len(p) > 0]
    M = len(items)
    if M == 0:
        return [], []
    paths, off = _pack([p for _, p in items], dg.device)
    total = int(off[-1].item())
    dev = dg.device
    tracks = torch.empty((max(total, 1), 3), dtype=torch.int32, device=dev)
    vias = torch.empty((max(total, 1), 3), dtype=torch.int32, device=dev)
    nt = torch.empty(M, dtype=torch.int32, device=dev)
    nv = torch.empty(M, dtype=torch.int32, device=dev)
    axis = np.array([1 if d == "h" else 2 for d in layer_dirs], np.int8)
    check(_lib.load().orsp_emit_geometry(dg.handle, M, ptr(paths), ptr(off), ptr(axis), ptr(tracks), ptr(vias),
                                         ptr(nt), ptr(nv), _stream()), "orsp_emit_geometry")
    off_h = off.cpu().numpy()
    nt_h, nv_h = nt.cpu().numpy(), nv.cpu().numpy()
    tr_h, vi_h = tracks.cpu().numpy(), vias.cpu().numpy()
    nx, plane = dg.nx, dg.nx * dg.ny

    def xy(node):
        r = np.asarray(node, np.int64) % plane
        return (_quantize(grid_min_x + (r % nx) * pitch, grid_min_x, pitch),
                _quantize(grid_min_y + (r // nx) * pitch, grid_min_y, pitch))

    def lname(z):
        return layer_names[z] if z < len(layer_names) else f"L{z}"

    out_t, out_v = [], []
    for m, (name, _) in enumerate(items):
        a = int(off_h[m])
        rows = tr_h[a:a + int(nt_h[m])]
        if len(rows):
            x1, y1 = xy(rows[:, 0])
            x2, y2 = xy(rows[:, 1])
            for i in range(len(rows)):
                out_t.append({"net": name, "layer": lname(int(rows[i, 2])), "x1": float(x1[i]), "y1": float(y1[i]),
                              "x2": float(x2[i]), "y2": float(y2[i]), "width": grid_pitch * 0.6})
        rows = vi_h[a:a + int(nv_h[m])]
        if len(rows):
            x, y = xy(rows[:, 0])
            for i in range(len(rows)):
                lo, hi = sorted((int(rows[i, 1]), int(rows[i, 2])))
                out_v.append({"net": name, "x": float(x[i]), "y": float(y[i]), "from_layer": lname(lo),
                              "to_layer": lname(hi), "diameter": 0.25, "drill": 0.15})
    return out_t, out_v
