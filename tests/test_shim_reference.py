"""install() on the unmodified reference router (CPU only, needs the
reference source tree; skipped where it is absent).  A stand-in solver that
answers through the oracle checks the wiring: every ROI search goes through
router.solver.gpu_solver and the routed result equals the reference's own
CPU run on the same lattice and nets (integer base costs, fp64 = fp32)."""
import os
from pathlib import Path

import numpy as np
import pytest

REF = Path(os.environ.get("ORTHOROUTE_REFERENCE", "/root/reference"))
pytestmark = pytest.mark.skipif(not (REF / "orthoroute").exists(), reason="reference source tree not available")


class _OracleSolver:
    """Stand-in for GpuSolver (test only): find_path_roi_gpu through the oracle."""

    def __init__(self, graph, lattice):
        self.indptr = np.asarray(graph.indptr)
        self.indices = np.asarray(graph.indices)
        self.calls = 0

    def find_path_roi_gpu(self, src, dst, costs, roi_nodes, global_to_roi):
        import oracle as O

        self.calls += 1
        p, *_ = O.dijkstra(self.indptr, self.indices, np.asarray(costs, np.float32), [int(src)], dst=int(dst),
                           roi_map=np.asarray(global_to_roi, np.int32))
        return p.tolist() if len(p) > 1 else None


def test_install_routes_every_roi_through_the_gpu_solver():
    from oracle.ref_harness import run_reference
    from orthoroute_b200.lattice import board_uniform_pins
    from orthoroute_b200.shim import install

    b = board_uniform_pins(20, 20, 4, 8, seed=2)
    base = run_reference(b.lattice, b.src, b.dst, ref=str(REF), max_iterations=3)
    holder = {}

    def factory(graph, lattice):
        holder["s"] = _OracleSolver(graph, lattice)
        return holder["s"]

    # run_reference builds the router; install after initialize_graph via a hook
    import oracle.ref_harness as H

    orig = H.run_reference

    def run_with_install(*a, **k):
        upf, _ = H._import(str(REF))
        real_init = upf.PathFinderRouter.initialize_graph

        def init(self, board):
            ok = real_init(self, board)
            install(self, path_to_edges=False, solver_factory=factory)
            return ok

        upf.PathFinderRouter.initialize_graph = init
        try:
            return orig(*a, **k)
        finally:
            upf.PathFinderRouter.initialize_graph = real_init

    got = run_with_install(b.lattice, b.src, b.dst, ref=str(REF), max_iterations=3)
    assert holder["s"].calls > 0
    assert got["trace"] == base["trace"]
    assert got["paths"] == base["paths"]
