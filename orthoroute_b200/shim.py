"""Installs the B200 search into an unmodified OrthoRoute PathFinderRouter.

The reference router already delegates ROI searches to ``router.solver.gpu_solver``
(orthoroute/algorithms/manhattan/unified_pathfinder.py, SimpleDijkstra.find_path_roi,
UPF:1801-1821) once the ROI is larger than ``gpu_roi_min_nodes``; ``install``
puts a ``GpuSolver`` there, lowers the threshold so that every ROI goes to the
GPU, and (optionally) replaces ``router._path_to_edges`` (UPF:5463) with the
device path -> edge mapping.  Nothing else in the router changes: net ordering,
rip-up, cost updates and the negotiation loop stay the reference's.
"""
from __future__ import annotations

from types import SimpleNamespace


def install(router, *, path_to_edges: bool = True, solver_factory=None, device=None):
    """Wires the GPU solver into `router` (after router.initialize_graph).

    solver_factory(graph, lattice) -> object with find_path_roi_gpu; defaults to
    orthoroute_b200.solver.GpuSolver (raises when no CUDA device is present -
    there is no CPU fallback).  Returns the solver."""
    if getattr(router, "graph", None) is None or getattr(router, "solver", None) is None:
        raise RuntimeError("install() needs an initialised router (call initialize_graph first)")
    if solver_factory is None:
        from .solver import GpuSolver

        def solver_factory(graph, lattice):
            return GpuSolver(graph, lattice, device=device)

    solver = solver_factory(router.graph, router.lattice)
    router.solver.gpu_solver = solver
    # SimpleDijkstra reads the threshold from self.config (UPF:1806)
    router.solver.config = SimpleNamespace(gpu_roi_min_nodes=0)
    if path_to_edges and hasattr(solver, "path_to_edges_list"):
        router._path_to_edges = solver.path_to_edges_list
    return solver
