"""install() wiring with the real CUDA solver, on a router-shaped object
(the reference tree is not needed): the solver lands in
router.solver.gpu_solver, searches match the oracle, a cost array rewritten
in place between calls is re-read, and router._path_to_edges matches the
oracle's path -> edge mapping."""
from types import SimpleNamespace

import numpy as np
import pytest

import oracle as O
from orthoroute_b200.lattice import build_lattice, uniform_weights
from orthoroute_b200.shim import install

pytestmark = pytest.mark.gpu


def _router(lat):
    return SimpleNamespace(graph=SimpleNamespace(indptr=lat.indptr, indices=lat.indices),
                           lattice=SimpleNamespace(x_steps=lat.nx, y_steps=lat.ny, layers=lat.nz),
                           solver=SimpleNamespace(gpu_solver=None, config=None),
                           _path_to_edges=None)


def test_install_solver_matches_oracle_and_sees_inplace_cost_updates():
    from orthoroute_b200.solver import GpuSolver

    lat = build_lattice(24, 20, 4)
    r = _router(lat)
    s = install(r)
    assert isinstance(r.solver.gpu_solver, GpuSolver) and s is r.solver.gpu_solver
    assert r.solver.config.gpu_roi_min_nodes == 0
    rng = np.random.default_rng(5)
    costs = uniform_weights(lat, 5).copy()
    N = lat.indptr.shape[0] - 1
    roi = np.arange(N, dtype=np.int32)
    g2r = roi.copy()
    for it in range(3):
        for _ in range(4):
            a, b = (int(v) for v in rng.integers(0, N, 2))
            got = s.find_path_roi_gpu(a, b, costs, roi, g2r)
            want, *_ = O.dijkstra(lat.indptr, lat.indices, costs, [a], dst=b)
            assert (got or []) == (want.tolist() if len(want) > 1 else [])
            e_got = r._path_to_edges(got or [])
            e_want = O.path_to_edges(lat.indptr, lat.indices, np.asarray(got or [], np.int32))
            assert e_got == e_want.tolist()
        # the router rewrites its cost array in place between iterations
        costs[:] = costs * np.float32(1.5) + rng.random(costs.shape[0], dtype=np.float32)
