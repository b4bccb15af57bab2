"""install() on the unmodified reference router (CPU only, needs the
reference source tree; skipped where it is absent).  A stand-in solver that
answers through the oracle checks the wiring: every ROI search goes through
router.solver.gpu_solver and the routed result equals the reference's own
CPU run on the same lattice and nets (integer base costs, fp64 = fp32)."""
import os
from pathlib import Path

import numpy as np
import pytest

# the reference source tree, named by ORTHOROUTE_REFERENCE (skipped when unset)
REF = Path(os.environ.get("ORTHOROUTE_REFERENCE") or "/nonexistent")
pytestmark = pytest.mark.skipif(not (REF / "orthoroute").exists(), reason="reference source tree not available")


class _OracleSolver:
    """Stand-in for GpuSolver (test only): find_path_roi_gpu through the
    oracle.  With `reference` (a SimpleDijkstra of the same graph) every
    search is also run by the reference's CPU Dijkstra on the same inputs;
    disagreements are counted, and so are those that are exact fp32 ties
    (both paths cost the same when their edge costs are added in fp32 in path
    order, as the search adds them)."""

    def __init__(self, graph, lattice, reference=None):
        self.indptr = np.asarray(graph.indptr)
        self.indices = np.asarray(graph.indices)
        self.reference = reference
        self.calls = self.diffs = self.ties = 0

    def _fp32_cost(self, path, c):
        import oracle as O

        d = np.float32(0)
        for e in O.path_to_edges(self.indptr, self.indices, np.asarray(path, np.int32)):
            d = np.float32(d + c[e])
        return d

    def find_path_roi_gpu(self, src, dst, costs, roi_nodes, global_to_roi):
        import oracle as O

        self.calls += 1
        c = np.asarray(costs, np.float32)
        p, *_ = O.dijkstra(self.indptr, self.indices, c, [int(src)], dst=int(dst),
                           roi_map=np.asarray(global_to_roi, np.int32))
        got = p.tolist() if len(p) > 1 else None
        if self.reference is not None:
            ref = self.reference.find_path_roi(int(src), int(dst), c, roi_nodes, global_to_roi)
            ref = list(map(int, ref)) if ref else None
            if got != ref:
                self.diffs += 1
                self.ties += int(got is not None and ref is not None and
                                 self._fp32_cost(got, c) == self._fp32_cost(ref, c))
        return got


@pytest.mark.parametrize("nx,ny,nz,nets,seed,iters", [(20, 20, 4, 8, 2, 3), (24, 18, 6, 14, 5, 4),
                                                       (18, 22, 4, 12, 7, 5), (22, 20, 6, 16, 9, 5),
                                                       (36, 30, 4, 120, 11, 3)])
def test_install_routes_every_roi_through_the_gpu_solver(nx, ny, nz, nets, seed, iters):
    """Every search of the run with the solver installed equals the reference
    CPU Dijkstra's on the same inputs, except exact fp32 ties.  Those arise
    when a path must cross an edge the reference blocks at a via keepout with
    cost 1e9 (_apply_via_keepouts_to_graph UPF:3067-3148, and the
    owner-aware keepouts of boards under 100 nets, UPF:3150-3241): the
    float32 sum absorbs the rest of the path, and the reference's float64
    sums break the tie differently.  A run without such a tie is the
    reference's own run, iteration for iteration and path for path."""
    import oracle.ref_harness as H
    from oracle.ref_harness import run_reference
    from orthoroute_b200.lattice import board_uniform_pins
    from orthoroute_b200.shim import install

    b = board_uniform_pins(nx, ny, nz, nets, seed=seed)
    base = run_reference(b.lattice, b.src, b.dst, ref=str(REF), max_iterations=iters)
    holder = {}

    def factory(graph, lattice):
        upf, _ = H._import(str(REF))
        holder["s"] = _OracleSolver(graph, lattice, reference=upf.SimpleDijkstra(graph, lattice=None))
        return holder["s"]

    # run_reference builds the router; install after initialize_graph via a hook

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

    got = run_with_install(b.lattice, b.src, b.dst, ref=str(REF), max_iterations=iters)
    s = holder["s"]
    assert s.calls > 0
    assert s.diffs == s.ties, f"{s.diffs - s.ties} searches differ without an fp32 tie"
    if s.diffs == 0:
        assert got["trace"] == base["trace"]
        assert got["paths"] == base["paths"]
