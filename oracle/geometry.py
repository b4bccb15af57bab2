"""ORACLE - test infrastructure only.

PathFinderRouter._generate_geometry_from_paths
(orthoroute/algorithms/manhattan/unified_pathfinder.py:5749-5834) restated in
plain Python on node indices: per net, the list of track runs (start node,
end node, layer) and vias (node, from layer, to layer) in emission order.
Pinned by tests/golden/golden_bookkeeping.npz.
"""
from __future__ import annotations


def emit(paths, nx, ny, nz, layer_dirs):
    plane = nx * ny
    out = []
    for path in paths:
        tracks, vias = [], []
        if len(path) == 0:
            out.append((tracks, vias))
            continue
        run_start = prev = int(path[0])
        prev_dir = None
        prev_layer = prev // plane
        for node in path[1:]:
            node = int(node)
            z0, r0 = divmod(prev, plane)
            z1, r1 = divmod(node, plane)
            y0, x0 = divmod(r0, nx)
            y1, x1 = divmod(r1, nx)
            if z0 == z1 and (z0 == 0 or z0 == nz - 1):
                prev, prev_layer, run_start = node, z1, node
                continue
            dx, dy, dz = abs(x1 - x0), abs(y1 - y0), abs(z1 - z0)
            if dz == 0:
                if dx + dy != 1:
                    continue
                if layer_dirs[z0] == "h":
                    if dy != 0:
                        continue
                elif dx != 0:
                    continue
            if z1 != z0:
                if prev != run_start:
                    tracks.append((run_start, prev, prev_layer))
                vias.append((prev, z0, z1))
                run_start = node
                prev_dir = None
            else:
                d = ((x1 > x0) - (x1 < x0), (y1 > y0) - (y1 < y0))
                if prev_dir is not None and d != prev_dir:
                    tracks.append((run_start, prev, prev_layer))
                    run_start = prev
                prev_dir = d
            prev, prev_layer = node, z1
        if prev != run_start:
            tracks.append((run_start, prev, prev_layer))
        out.append((tracks, vias))
    return out
