"""Device graph and the GPU solver with the reference's gpu_solver interface.

``DeviceGraph`` owns the uploaded CSR (through liborsp.so) and exposes the
kernels as methods on torch CUDA tensors.  ``GpuSolver`` is the object the
reference router expects in ``router.solver.gpu_solver``
(orthoroute/algorithms/manhattan/unified_pathfinder.py:2199-2218): the same
method names, arguments and return conventions as CUDADijkstra
(orthoroute/algorithms/manhattan/pathfinder/cuda_dijkstra.py), with the exact
fp32 semantics of SimpleDijkstra.find_path_roi (UPF:1801-1887).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr

DEFAULT_PATH_CAP = 1 << 16


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("orthoroute_b200 needs a CUDA device (sm_100a); no CPU fallback exists")


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


def as_device(a, dtype, device) -> torch.Tensor:
    """numpy / list / tensor -> contiguous CUDA tensor of `dtype` (no copy when
    it already is one)."""
    if isinstance(a, torch.Tensor):
        t = a
        if t.device != device or t.dtype != dtype:
            t = t.to(device=device, dtype=dtype)
        return t.contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype=torch.empty(0, dtype=dtype).numpy().dtype)
    return torch.from_numpy(arr).to(device)


class DeviceGraph:
    """CSR graph resident on one GPU (forward CSR + transposed CSR)."""

    def __init__(self, indptr, indices, nx: int = 0, ny: int = 0, nz: int = 0, device=None):
        _require_cuda()
        lib = _lib.load()
        dev = torch.device(device) if device is not None else torch.device("cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.N = int(indptr.shape[0] - 1)
        self.E = int(indices.shape[0])
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(lib.orsp_graph_create(self.N, self.E, ptr(indptr), ptr(indices), self.nx, self.ny,
                                        self.nz, self.device.index or 0, ctypes.byref(h)),
                  "orsp_graph_create")
        self._h = h
        md = ctypes.c_int32()
        check(lib.orsp_graph_max_degree(self._h, ctypes.byref(md)), "orsp_graph_max_degree")
        self.max_degree = int(md.value)
        self.indptr_host = indptr
        self.indices_host = indices
        self._path_buf = None
        self._edge_buf = None
        self._g2r_buf = None

    @classmethod
    def from_lattice(cls, lat, device=None) -> "DeviceGraph":
        return cls(lat.indptr, lat.indices, lat.nx, lat.ny, lat.nz, device=device)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().orsp_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ utils
    def _path_buffer(self, cap: int) -> torch.Tensor:
        if self._path_buf is None or self._path_buf.numel() < cap:
            self._path_buf = torch.empty(cap, dtype=torch.int32, device=self.device)
        return self._path_buf

    @staticmethod
    def default_delta(cost: torch.Tensor) -> float:
        """Bucket width: twice the mean of a strided sample of finite costs."""
        n = cost.numel()
        step = max(1, n // 65536)
        s = cost[::step]
        s = s[torch.isfinite(s)]
        if s.numel() == 0:
            return 1.0
        m = float(s.mean())
        return max(2.0 * m, 1e-6)

    # --------------------------------------------------------------- searches
    def sssp(self, cost: torch.Tensor, seeds, dst: int = -1, roi_map: Optional[torch.Tensor] = None,
             seed_cost: Optional[torch.Tensor] = None, delta: Optional[float] = None,
             dist_out: Optional[torch.Tensor] = None, path_cap: Optional[int] = None):
        """Runs the persistent grid search.  Returns (status, path tensor (device,
        int32, possibly empty), rounds)."""
        lib = _lib.load()
        seeds_t = as_device(np.atleast_1d(seeds) if not isinstance(seeds, torch.Tensor) else seeds,
                            torch.int32, self.device)
        if delta is None:
            delta = self.default_delta(cost)
        cap = int(path_cap or min(self.N + 1, DEFAULT_PATH_CAP))
        pbuf = self._path_buffer(cap) if dst >= 0 else None
        plen = ctypes.c_int32(0)
        rounds = ctypes.c_int32(0)
        st = check(lib.orsp_sssp(self._h, ptr(cost), int(seeds_t.numel()), ptr(seeds_t), ptr(seed_cost),
                                 int(dst), ptr(roi_map), float(delta), ptr(dist_out), ptr(pbuf), cap,
                                 ctypes.byref(plen), ctypes.byref(rounds), _stream()), "orsp_sssp")
        path = pbuf[: plen.value] if (dst >= 0 and st == _lib.ORSP_OK) else None
        return st, path, int(rounds.value)

    def batch_bbox(self, cost: torch.Tensor, src: torch.Tensor, dst: torch.Tensor, bbox: torch.Tensor,
                   order: Optional[torch.Tensor] = None, delta: Optional[float] = None,
                   path_cap: int = 4096, with_edges: bool = True):
        """K box-ROI searches in one launch.  Returns (nodes[K,cap], edges[K,cap]
        or None, lens[K]) as device tensors; lens < 2 means no path."""
        lib = _lib.load()
        K = int(src.numel())
        if delta is None:
            delta = self.default_delta(cost)
        nodes = torch.empty((K, path_cap), dtype=torch.int32, device=self.device)
        edges = torch.empty((K, path_cap), dtype=torch.int32, device=self.device) if with_edges else None
        lens = torch.zeros(K, dtype=torch.int32, device=self.device)
        check(lib.orsp_sssp_batch_bbox(self._h, ptr(cost), K, ptr(src), ptr(dst), ptr(bbox), ptr(order),
                                       float(delta), ptr(nodes), ptr(edges), int(path_cap), ptr(lens),
                                       _stream()), "orsp_sssp_batch_bbox")
        return nodes, edges, lens

    def roi_bfs(self, src: int, dst: int, max_depth: int, max_nodes: int = 50_000, want_g2r: bool = True):
        """Bidirectional BFS ROI.  Returns (roi_nodes device int32[R], g2r device int32[N] or None)."""
        lib = _lib.load()
        roi = torch.empty(self.N, dtype=torch.int32, device=self.device)
        g2r = torch.empty(self.N, dtype=torch.int32, device=self.device) if want_g2r else None
        cnt = ctypes.c_int32(0)
        check(lib.orsp_roi_bfs(self._h, int(src), int(dst), int(max_depth), int(max_nodes), ptr(roi),
                               ptr(g2r), ctypes.byref(cnt), _stream()), "orsp_roi_bfs")
        return roi[: cnt.value], g2r

    def path_to_edges(self, path: torch.Tensor) -> torch.Tensor:
        lib = _lib.load()
        n = int(path.numel())
        out = torch.empty(max(n - 1, 1), dtype=torch.int32, device=self.device)
        cnt = ctypes.c_int32(0)
        check(lib.orsp_path_to_edges(self._h, ptr(path), n, ptr(out), ctypes.byref(cnt), _stream()),
              "orsp_path_to_edges")
        return out[: cnt.value]


class GpuSolver:
    """Drop-in for ``router.solver.gpu_solver`` (CUDADijkstra's interface)."""

    def __init__(self, graph=None, lattice=None, device=None):
        _require_cuda()
        if isinstance(graph, DeviceGraph):
            self.dg = graph
        else:
            indptr = graph.indptr.get() if hasattr(graph.indptr, "get") else np.asarray(graph.indptr)
            indices = graph.indices.get() if hasattr(graph.indices, "get") else np.asarray(graph.indices)
            nx = getattr(lattice, "x_steps", 0) if lattice is not None else 0
            ny = getattr(lattice, "y_steps", 0) if lattice is not None else 0
            nz = getattr(lattice, "layers", 0) if lattice is not None else 0
            self.dg = DeviceGraph(indptr, indices, nx, ny, nz, device=device)
        self.lattice = lattice
        self.N = self.dg.N
        self._cost_cache = (None, None)

    def _cost(self, costs) -> torch.Tensor:
        if isinstance(costs, torch.Tensor) and costs.is_cuda:
            return as_device(costs, torch.float32, self.dg.device)
        key = id(costs)
        if self._cost_cache[0] == key:
            return self._cost_cache[1]
        t = as_device(costs, torch.float32, self.dg.device)
        self._cost_cache = (key, t)
        return t

    def find_path_roi_gpu(self, src: int, dst: int, costs, roi_nodes, global_to_roi) -> Optional[List[int]]:
        """CUDADijkstra.find_path_roi_gpu (CD:4909): node path src..dst in global
        ids, or None.  Semantics of SimpleDijkstra.find_path_roi: the search is
        restricted to nodes with global_to_roi >= 0 and ties between equal
        distances go to the smaller ROI index."""
        cost = self._cost(costs)
        n_roi = len(roi_nodes)
        full = n_roi == self.N and int(roi_nodes[0]) == 0 and int(roi_nodes[-1]) == self.N - 1
        g2r = None if full else as_device(global_to_roi, torch.int32, self.dg.device)
        if g2r is not None and (int(global_to_roi[src]) < 0 or int(global_to_roi[dst]) < 0):
            return None
        st, path, _ = self.dg.sssp(cost, int(src), int(dst), roi_map=g2r)
        if st != _lib.ORSP_OK or path is None or path.numel() < 2:
            return None
        return path.cpu().tolist()
