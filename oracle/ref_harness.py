"""ORACLE - test infrastructure only: runs the unmodified reference router
(OrthoRoute's PathFinderRouter, CPU path) on a synthetic lattice.

Only usable where the reference source tree is available (it is not shipped
with this repository).  The harness follows the pinning rules needed to run
the reference at fixed parameters:

* the lattice CSR is injected by replacing Lattice3D.build_graph
  (orthoroute/algorithms/manhattan/unified_pathfinder.py:1180, "UPF") so that
  the router searches exactly the benchmark graph;
* apply_derived_parameters (parameter_derivation.py:204-264) is replaced by a
  no-op, so pres_fac_init / max_iterations stay as configured;
* ORTHO_PRES_FAC_MULT / ORTHO_HIST_GAIN pin the schedule (UPF:3588-3590);
* random.seed is set before routing (iteration 1 uses the global random
  module, UPF:4434).
Optionally SimpleDijkstra.find_path_roi is replaced by a callable (e.g. the
fp32 oracle) to record the reference loop with fp32 search semantics.
"""
from __future__ import annotations

import logging
import os
import random
import sys
import time
from types import SimpleNamespace

import numpy as np


def _import(ref):
    sys.dont_write_bytecode = True
    if ref not in sys.path:
        sys.path.insert(0, ref)
    logging.disable(logging.CRITICAL)
    import orthoroute.algorithms.manhattan.unified_pathfinder as upf
    import orthoroute.algorithms.manhattan.parameter_derivation as pd

    return upf, pd


def reference_root(ref=None) -> str:
    """The OrthoRoute source tree: `ref`, else $ORTHOROUTE_REFERENCE."""
    ref = ref or os.environ.get("ORTHOROUTE_REFERENCE")
    if not ref:
        raise RuntimeError("set ORTHOROUTE_REFERENCE to the OrthoRoute source tree (or pass ref=)")
    return ref


def run_reference(lat, src, dst, *, ref=None, max_iterations=30, pres_fac_init=0.5,
                  pres_fac_mult=1.5, hist_gain=1.0, seed=0, search=None, record=None, on_init=None,
                  on_iteration=None):
    """Routes nets (src[i] -> dst[i]) with the reference router.

    search: optional callable(indptr, indices, src, dst, costs, roi_nodes, g2r) -> path list or None
            that replaces SimpleDijkstra.find_path_roi.
    record: optional list; receives one dict per search call
            (iteration, src, dst, costs-id, roi_nodes, path).
    on_init: optional callable(router), called after initialize_graph.
    on_iteration: optional callable(it, over_sum, over_cnt) after each iteration.
    Returns dict(result, trace=[(it, over_sum, over_cnt)], paths, seconds)."""
    upf, pd = _import(reference_root(ref))
    os.environ["ORTHO_PRES_FAC_MULT"] = repr(float(pres_fac_mult))
    os.environ["ORTHO_HIST_GAIN"] = repr(float(hist_gain))
    pitch = 0.5

    def build_graph(self, via_cost, allowed_via_spans=None, use_gpu=False):
        g = upf.CSRGraph(False)
        g.indptr = lat.indptr.copy()
        g.indices = lat.indices.copy()
        g.base_costs = lat.base_cost.copy()
        g.edge_layer = lat.edge_layer.copy()
        g.edge_kind = lat.edge_kind.copy()
        return g

    saved = (upf.Lattice3D.build_graph, upf.apply_derived_parameters, upf.SimpleDijkstra.find_path_roi)
    upf.Lattice3D.build_graph = build_graph
    upf.apply_derived_parameters = lambda cfg, params: None
    if search is not None:
        def find_path_roi(self, s, d, costs, roi_nodes, global_to_roi):
            p = search(self.indptr, self.indices, s, d, costs, roi_nodes, global_to_roi)
            if record is not None:
                record.append({"src": int(s), "dst": int(d), "roi": np.asarray(roi_nodes, dtype=np.int32).copy(),
                               "costs": np.asarray(costs, dtype=np.float32), "path": list(p) if p else []})
            return p
        upf.SimpleDijkstra.find_path_roi = find_path_roi
    try:
        cfg = upf.PathFinderConfig()
        cfg.use_gpu = False
        cfg.portal_enabled = False
        cfg.grid_pitch = pitch
        cfg.max_iterations = max_iterations
        cfg.pres_fac_init = pres_fac_init
        cfg.pres_fac_mult = pres_fac_mult
        cfg.hist_gain = hist_gain
        cfg.layer_count = lat.nz
        pos = lambda x, y: SimpleNamespace(x=x, y=y)  # noqa: E731
        margin = 3.0
        p1 = SimpleNamespace(position=pos(margin, margin), layer="F.Cu", net_name="BOUNDS", id="b1")
        p2 = SimpleNamespace(position=pos((lat.nx - 1) * pitch - margin, (lat.ny - 1) * pitch - margin),
                             layer="F.Cu", net_name="BOUNDS", id="b2")
        board = SimpleNamespace(nets=[SimpleNamespace(name="BOUNDS", pads=[p1, p2])], components=[], pads=[],
                                layer_count=lat.nz, layers=None)
        router = upf.PathFinderRouter(cfg, use_gpu=False)
        router.initialize_graph(board)
        assert router.lattice.x_steps == lat.nx and router.lattice.y_steps == lat.ny, "lattice injection failed"
        if on_init is not None:
            on_init(router)
        trace = []

        def it_cb(it, tracks, vias, over_sum, over_cnt):
            trace.append((it, int(over_sum), int(over_cnt)))
            if on_iteration is not None:
                on_iteration(it, over_sum, over_cnt)

        reqs = [(f"N{i}", int(s), int(d)) for i, (s, d) in enumerate(zip(src, dst))]
        random.seed(seed)
        t0 = time.perf_counter()
        res = router.route_multiple_nets(reqs, iteration_cb=it_cb)
        secs = time.perf_counter() - t0
        paths = {k: list(v) for k, v in router.net_paths.items()}
        return {"result": res, "trace": trace, "paths": paths, "seconds": secs, "router": router}
    finally:
        upf.Lattice3D.build_graph, upf.apply_derived_parameters, upf.SimpleDijkstra.find_path_roi = saved
