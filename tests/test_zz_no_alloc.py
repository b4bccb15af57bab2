"""orsp_roi_bfs_noalloc: ROI extraction for callers that cannot allocate device
memory while they route (an application whose own caching allocator has
reserved the GPU's memory and allows no other cudaMalloc / cudaFree on the
routing path).  Its work buffers are one fixed array inside the library; the
results must equal those of the allocating entry point orsp_roi_bfs, call
after call.

This file is collected last on purpose, so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from orthoroute_b200 import _lib  # noqa: E402
from orthoroute_b200.lattice import build_lattice  # noqa: E402
from orthoroute_b200.solver import DeviceGraph  # noqa: E402

MAX_NODES = 524288  # ORSP_ROI_BFS_NOALLOC_MAX_NODES in include/orsp.h


def _extract(fn, dg, src, dst, depth, max_nodes):
    roi = torch.full((dg.N,), -7, dtype=torch.int32, device=dg.device)
    g2r = torch.full((dg.N,), -7, dtype=torch.int32, device=dg.device)
    cnt = ctypes.c_int32(-1)
    stream = int(torch.cuda.current_stream().cuda_stream)
    rc = fn(dg.handle, src, dst, depth, max_nodes, _lib.ptr(roi), _lib.ptr(g2r), ctypes.byref(cnt), stream)
    torch.cuda.synchronize()
    return rc, roi[: max(cnt.value, 0)].cpu().numpy(), g2r.cpu().numpy()


def test_noalloc_roi_matches_allocating_entry_point_on_consecutive_calls():
    lib = _lib.load()
    lat = build_lattice(150, 120, 6)  # 108 000 nodes
    assert lat.N <= MAX_NODES
    dg = DeviceGraph.from_lattice(lat)
    rng = np.random.default_rng(12)
    # consecutive calls: a large ROI, then a small truncated one, then a
    # large one again (the array keeps the previous call's contents)
    cases = [(60, 50_000), (9, 700), (150, 50_000)]
    for depth, max_nodes in cases:
        s, d = (int(v) for v in rng.choice(lat.N, size=2, replace=False))
        rc_na, roi_na, g2r_na = _extract(lib.orsp_roi_bfs_noalloc, dg, s, d, depth, max_nodes)
        rc, roi, g2r = _extract(lib.orsp_roi_bfs, dg, s, d, depth, max_nodes)
        assert rc_na == rc == _lib.ORSP_OK, lib.orsp_last_error()
        assert np.array_equal(roi_na, roi)
        assert np.array_equal(g2r_na, g2r)
        assert len(roi_na) > 0 and s in set(roi_na.tolist()) and d in set(roi_na.tolist())


def test_noalloc_roi_at_the_array_limit():
    """A graph of exactly ORSP_ROI_BFS_NOALLOC_MAX_NODES nodes fills the visit
    marks, queues and compaction tiles to their ends."""
    lib = _lib.load()
    lat = build_lattice(1024, 256, 2)  # 524 288 nodes, both axes on both layers
    assert lat.N == MAX_NODES
    dg = DeviceGraph.from_lattice(lat)
    # deep searches from the two ends of the node range (the last node and
    # the last compaction tile are marked), a shallow one between them
    for s, d, depth, max_nodes in ((0, lat.N - 1, 150, MAX_NODES), (77, 5000, 12, 900),
                                   (lat.N - 1, 0, 150, MAX_NODES)):
        rc_na, roi_na, g2r_na = _extract(lib.orsp_roi_bfs_noalloc, dg, s, d, depth, max_nodes)
        rc, roi, g2r = _extract(lib.orsp_roi_bfs, dg, s, d, depth, max_nodes)
        assert rc_na == rc == _lib.ORSP_OK, lib.orsp_last_error()
        assert np.array_equal(roi_na, roi)
        assert np.array_equal(g2r_na, g2r)


def test_noalloc_roi_rejects_graphs_beyond_its_array():
    lib = _lib.load()
    lat = build_lattice(1024, 520, 1)  # 532 480 nodes
    assert lat.N > MAX_NODES
    dg = DeviceGraph.from_lattice(lat)
    rc, _, _ = _extract(lib.orsp_roi_bfs_noalloc, dg, 0, 5, 4, 1000)
    assert rc == _lib.ORSP_ERR_ARG
    assert b"orsp_roi_bfs" in lib.orsp_last_error()
