"""Golden vectors for the per-iteration negotiation bookkeeping, produced by
the reference's own methods on a real router state.

    python tests/golden/make_golden_bookkeeping.py [--ref <OrthoRoute tree>]  (default: $ORTHOROUTE_REFERENCE)

A small board is routed for a few iterations by the unmodified reference
router (oracle/ref_harness.py), then, on that router's state:

  PathFinderRouter._rebuild_node_owner            UPF:2762-2837  -> node_owner
  PathFinderRouter._detect_barrel_conflicts       UPF:5478-5569  -> conflict edges
  the barrel penalty of _pathfinder_negotiation   UPF:3852-3871  -> present after
  PathFinderRouter._order_nets_by_difficulty      UPF:4401-4439  -> net order
  PathFinderRouter._build_hotset                  UPF:5009-5140  -> hotset
  PathFinderRouter._generate_geometry_from_paths  UPF:5749-5897  -> tracks, vias

Output: golden_bookkeeping.npz (UPF = orthoroute/algorithms/manhattan/
unified_pathfinder.py).  Net names are stored by index (net k is "N{k}").
"""
from __future__ import annotations

import argparse
import os
import random
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ORTHOROUTE_REFERENCE"),
                    required=not os.environ.get("ORTHOROUTE_REFERENCE"),
                    help="OrthoRoute source tree (default: $ORTHOROUTE_REFERENCE)")
    args = ap.parse_args()
    from oracle.ref_harness import run_reference
    from orthoroute_b200.lattice import board_uniform_pins

    out = {}
    cases = [(40, 36, 6, 70, 5, 4), (32, 30, 4, 45, 9, 3)]
    out["ncases"] = np.int32(len(cases))
    for c, (nx, ny, nz, nets, seed, iters) in enumerate(cases):
        b = board_uniform_pins(nx, ny, nz, nets, seed=seed)
        res = run_reference(b.lattice, b.src, b.dst, ref=args.ref, max_iterations=iters)
        r = res["router"]
        names = [f"N{k}" for k in range(nets)]
        N = b.lattice.N
        # net paths and edge lists in the router's dict order
        order = [n for n in r.net_paths.keys()]
        paths = [list(r.net_paths[n]) for n in order]
        edges = [list(r._net_to_edges.get(n, [])) for n in order]
        pfx = f"c{c}_"
        out[pfx + "dims"] = np.array([nx, ny, nz], np.int32)
        out[pfx + "board"] = np.array([nx, ny, nz, nets, seed], np.int32)  # board_uniform_pins arguments
        out[pfx + "order"] = np.array([names.index(n) for n in order], np.int32)
        out[pfx + "plen"] = np.array([len(p) for p in paths], np.int32)
        out[pfx + "paths"] = np.array([v for p in paths for v in p], np.int32)
        out[pfx + "elen"] = np.array([len(e) for e in edges], np.int32)
        out[pfx + "edges"] = np.array([v for e in edges for v in e], np.int32)
        # escape-via keepouts (z, x, y) -> net, in dict order (first owner wins)
        keep = list(getattr(r, "_via_keepouts_map", {}).items())
        out[pfx + "keepouts"] = np.array([[z, x, y, names.index(n)] for (z, x, y), n in keep], np.int32).reshape(-1, 4)
        # node ownership (net ids assigned on first use, in dict order)
        r.net_id_map = {}
        r.next_net_id = 0
        r._rebuild_node_owner()
        out[pfx + "node_owner"] = r.node_owner.copy()
        out[pfx + "net_ids"] = np.array([r.net_id_map.get(n, -1) for n in names], np.int32)
        conf, cnt = r._detect_barrel_conflicts()
        out[pfx + "conflicts"] = np.asarray(conf, np.int32)
        out[pfx + "conflict_count"] = np.int32(cnt)
        pres_fac = 3.375
        present = np.asarray(r.accounting.present, dtype=np.float32).copy()
        out[pfx + "present"] = present.copy()
        penalty = min(10.0 * pres_fac, 100.0)
        present[np.asarray(conf, dtype=np.int64)] += penalty
        out[pfx + "present_after"] = present
        out[pfx + "pres_fac"] = np.float32(pres_fac)
        out[pfx + "capacity"] = np.asarray(r.accounting.capacity, dtype=np.float32).copy()
        out[pfx + "history"] = np.asarray(r.accounting.history, dtype=np.float32).copy()
        # difficulty order (its shuffle draws from the global random module)
        tasks = {names[k]: (int(b.src[k]), int(b.dst[k])) for k in range(nets)}
        random.seed(17 + c)
        ordered = r._order_nets_by_difficulty(tasks)
        out[pfx + "difficulty_order"] = np.array([names.index(n) for n in ordered], np.int32)
        out[pfx + "shuffle_seed"] = np.int32(17 + c)
        # hotset, from a fixed bookkeeping state
        r.iteration = 6 + c
        r._net_clean_iters = {names[k]: (k % 5) for k in range(nets)}
        r._last_reroute_iter = {names[k]: r.iteration - 1 for k in range(0, nets, 7)}
        clean_before = dict(r._net_clean_iters)
        last_before = dict(r._last_reroute_iter)
        hot = r._build_hotset(tasks, ripped={names[1]})
        out[pfx + "hot_iteration"] = np.int32(r.iteration)
        out[pfx + "hot_clean_before"] = np.array([clean_before.get(n, 0) for n in names], np.int32)
        out[pfx + "hot_last_before"] = np.array([last_before.get(n, -999) for n in names], np.int32)
        out[pfx + "hot_cap"] = np.int32(r.config.hotset_cap)
        out[pfx + "hotset"] = np.array(sorted(names.index(n) for n in hot), np.int32)
        out[pfx + "hot_clean_after"] = np.array([r._net_clean_iters.get(n, 0) for n in names], np.int32)
        # geometry of the committed paths (world coordinates, layer indices)
        tracks, vias = r._generate_geometry_from_paths()
        lnames = list(r.config.layer_names)
        lidx = lambda nm: lnames.index(nm) if nm in lnames else int(nm[1:])  # noqa: E731
        out[pfx + "tracks"] = np.array([[names.index(t["net"]), lidx(t["layer"])] for t in tracks],
                                       np.int32).reshape(-1, 2)
        out[pfx + "track_xy"] = np.array([[t["x1"], t["y1"], t["x2"], t["y2"]] for t in tracks],
                                         np.float64).reshape(-1, 4)
        out[pfx + "vias"] = np.array([[names.index(v["net"]), lidx(v["from_layer"]), lidx(v["to_layer"])]
                                      for v in vias], np.int32).reshape(-1, 3)
        out[pfx + "via_xy"] = np.array([[v["x"], v["y"]] for v in vias], np.float64).reshape(-1, 2)
        geom = r.lattice.geom
        out[pfx + "geom"] = np.array([geom.grid_min_x, geom.grid_min_y, geom.pitch], np.float64)
        out[pfx + "layer_names"] = np.array(lnames)
        out[pfx + "layer_dir"] = np.array([r.lattice.get_legal_axis(z) for z in range(nz)])
        print(f"case {c}: {len(order)} routed nets, owned nodes {(r.node_owner >= 0).sum()}, conflicts {cnt}, "
              f"hotset {len(hot)}, tracks {len(tracks)}, vias {len(vias)}")
    np.savez_compressed(HERE / "golden_bookkeeping.npz", **out)


if __name__ == "__main__":
    main()
