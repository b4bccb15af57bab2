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
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from ._lib import load as _load_lib

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
        il = ctypes.c_int32()
        check(lib.orsp_graph_is_lattice(self._h, ctypes.byref(il)), "orsp_graph_is_lattice")
        # 1: H/V lattice with adjacent-layer vias; 2: the same with column
        # vias (the reference's Lattice3D), searched with a per-column via pass
        self.lattice_kind = int(il.value)
        self.is_lattice = self.lattice_kind != 0
        ml = ctypes.c_int32()
        check(lib.orsp_lattice_max_layers(0, ctypes.byref(ml)), "orsp_lattice_max_layers")
        # the device routing loop needs every box in one shared-memory tile
        self.route_loop_ok = self.is_lattice and self.nz <= int(ml.value)
        self.indptr_host = indptr
        self.indices_host = indices
        self._path_buf = None
        self._edge_buf = None
        self._g2r_buf = None
        self._seed_buf = None

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

    # --------------------------------------------------------------- searches
    def sssp(self, cost: torch.Tensor, seeds, dst: int = -1, roi_map: Optional[torch.Tensor] = None,
             seed_cost: Optional[torch.Tensor] = None, delta: Optional[float] = None,
             dist_out: Optional[torch.Tensor] = None, path_cap: Optional[int] = None,
             cost_generation: Optional[int] = None):
        """One search (orsp_sssp: the lattice tile sweep or the generic grid
        search).  cost_generation (non-zero): the caller's identifier of the
        cost array's current contents, declared for this search
        (orsp_graph_cost_generation); a whole-lattice search then reuses the
        weights gathered by an earlier search with the same array and
        generation.  Returns (status, path tensor (device, int32, possibly
        empty), rounds)."""
        lib = _lib.load()
        if cost_generation:
            check(lib.orsp_graph_cost_generation(self._h, ptr(cost), int(cost_generation)),
                  "orsp_graph_cost_generation")
        if isinstance(seeds, (int, np.integer)):
            # one seed: a device fill instead of a host->device copy
            if self._seed_buf is None:
                self._seed_buf = torch.empty(1, dtype=torch.int32, device=self.device)
            seeds_t = self._seed_buf.fill_(int(seeds))
        else:
            seeds_t = as_device(np.atleast_1d(seeds) if not isinstance(seeds, torch.Tensor) else seeds,
                                torch.int32, self.device)
        if delta is None:
            delta = 0.0  # chosen on the device
        cap = int(path_cap or min(self.N + 1, DEFAULT_PATH_CAP))
        pbuf = self._path_buffer(cap) if dst >= 0 else None
        plen = ctypes.c_int32(0)
        rounds = ctypes.c_int32(0)
        st = check(lib.orsp_sssp(self._h, ptr(cost), int(seeds_t.numel()), ptr(seeds_t), ptr(seed_cost),
                                 int(dst), ptr(roi_map), float(delta), ptr(dist_out), ptr(pbuf), cap,
                                 ctypes.byref(plen), ctypes.byref(rounds), _stream()), "orsp_sssp")
        path = pbuf[: plen.value] if (dst >= 0 and st == _lib.ORSP_OK) else None
        return st, path, int(rounds.value)

    def sssp_sources(self, cost: torch.Tensor, sources, dist_out: torch.Tensor, per_launch: int = 0,
                     cost_generation: Optional[int] = None) -> int:
        """Full searches from every source (orsp_sssp_sources): row i of
        dist_out (device fp32 [len(sources), N]) receives the distances from
        sources[i]; on a lattice up to per_launch sources (0: all) share one
        launch.  Returns the status."""
        lib = _lib.load()
        src = np.ascontiguousarray(np.asarray(sources, dtype=np.int32).ravel())
        if dist_out.dtype != torch.float32 or not dist_out.is_contiguous() or dist_out.numel() != src.size * self.N:
            raise ValueError("dist_out must be a contiguous float32 tensor of len(sources) * N")
        if cost_generation:
            check(lib.orsp_graph_cost_generation(self._h, ptr(cost), int(cost_generation)),
                  "orsp_graph_cost_generation")
        return check(lib.orsp_sssp_sources(self._h, ptr(cost), int(src.size),
                                           src.ctypes.data_as(ctypes.c_void_p), ptr(dist_out), int(per_launch),
                                           _stream()), "orsp_sssp_sources")

    def sssp_roi_nodes(self, cost: torch.Tensor, src: int, dst: int, roi_nodes: torch.Tensor,
                       path_cap: Optional[int] = None):
        """One search src -> dst over the ROI given as its node list (device
        int32; ROI index = position).  Returns (status, path tensor or None)."""
        lib = _lib.load()
        cap = int(path_cap or min(self.N + 1, DEFAULT_PATH_CAP))
        pbuf = self._path_buffer(cap)
        plen = ctypes.c_int32(0)
        st = check(lib.orsp_sssp_roi_nodes(self._h, ptr(cost), int(src), int(dst), ptr(roi_nodes),
                                           int(roi_nodes.numel()), ptr(pbuf), cap, ctypes.byref(plen), _stream()),
                   "orsp_sssp_roi_nodes")
        path = pbuf[: plen.value] if st == _lib.ORSP_OK else None
        return st, path

    def sssp_box(self, cost: torch.Tensor, src: int, dst: int, box, delta: Optional[float] = None,
                 dist_out: Optional[torch.Tensor] = None, path_cap: Optional[int] = None):
        """One search inside the inclusive box (x0, x1, y0, y1, z0, z1): the
        result of sssp() with the box's ROI map, without building the map.
        Returns (status, path tensor or None, rounds)."""
        lib = _lib.load()
        if self._seed_buf is None:
            self._seed_buf = torch.empty(1, dtype=torch.int32, device=self.device)
        seeds_t = self._seed_buf.fill_(int(src))
        bx = (ctypes.c_int32 * 6)(*[int(v) for v in box])
        cap = int(path_cap or min(self.N + 1, DEFAULT_PATH_CAP))
        pbuf = self._path_buffer(cap) if dst >= 0 else None
        plen = ctypes.c_int32(0)
        rounds = ctypes.c_int32(0)
        st = check(lib.orsp_sssp_box(self._h, ptr(cost), 1, ptr(seeds_t), None, int(dst), bx,
                                     float(0.0 if delta is None else delta), ptr(dist_out), ptr(pbuf), cap,
                                     ctypes.byref(plen), ctypes.byref(rounds), _stream()), "orsp_sssp_box")
        path = pbuf[: plen.value] if (dst >= 0 and st == _lib.ORSP_OK) else None
        return st, path, int(rounds.value)

    def sssp_multi(self, cost: torch.Tensor, seeds, targets, seed_cost=None, target_cost=None,
                   roi_map: Optional[torch.Tensor] = None, delta: Optional[float] = None,
                   path_cap: Optional[int] = None):
        """Exact multi-seed / multi-target search (targets are sinks).  Returns
        (status, path tensor or None, best target id)."""
        lib = _load_lib()
        seeds_t = as_device(np.atleast_1d(seeds) if not isinstance(seeds, torch.Tensor) else seeds, torch.int32,
                            self.device)
        tg = as_device(np.atleast_1d(targets) if not isinstance(targets, torch.Tensor) else targets, torch.int32,
                       self.device)
        sc = None if seed_cost is None else as_device(seed_cost, torch.float32, self.device)
        tc = None if target_cost is None else as_device(target_cost, torch.float64, self.device)
        if delta is None:
            delta = 0.0  # chosen on the device
        cap = int(path_cap or min(self.N + 1, DEFAULT_PATH_CAP))
        pbuf = self._path_buffer(cap)
        plen = ctypes.c_int32(0)
        best = ctypes.c_int32(-1)
        st = check(lib.orsp_sssp_multi(self._h, ptr(cost), int(seeds_t.numel()), ptr(seeds_t), ptr(sc),
                                       int(tg.numel()), ptr(tg), ptr(tc), ptr(roi_map), float(delta), ptr(pbuf), cap,
                                       ctypes.byref(plen), ctypes.byref(best), _stream()), "orsp_sssp_multi")
        path = pbuf[: plen.value] if st == _lib.ORSP_OK else None
        return st, path, int(best.value)

    def roi_from_bitmap(self, bitmap) -> torch.Tensor:
        bm = as_device(bitmap, torch.int32, self.device) if not isinstance(bitmap, torch.Tensor) else bitmap
        g2r = torch.empty(self.N, dtype=torch.int32, device=self.device)
        check(_load_lib().orsp_roi_from_bitmap(self._h, ptr(bm), ptr(g2r), _stream()), "orsp_roi_from_bitmap")
        return g2r

    def set_batch_plan(self, buckets=None):
        """Tuning plan of batch_bbox: a list of dicts {max_nodes, impl (0: one
        CTA per search, 1: tile sweeps), delta (0: the call's), tile_w,
        ctas_per_sm (0: default)}, by increasing max_nodes; None or [] restores
        the default.  The paths do not depend on the plan."""
        buckets = buckets or []
        n = len(buckets)
        mx = np.array([int(b["max_nodes"]) for b in buckets], dtype=np.int64)
        im = np.array([int(b.get("impl", 0)) for b in buckets], dtype=np.int32)
        de = np.array([float(b.get("delta", 0.0)) for b in buckets], dtype=np.float32)
        tw = np.array([int(b.get("tile_w", 16)) for b in buckets], dtype=np.int32)
        cp = np.array([int(b.get("ctas_per_sm", 0)) for b in buckets], dtype=np.int32)
        check(_lib.load().orsp_batch_set_plan(self._h, n, ptr(mx) if n else None, ptr(im) if n else None,
                                              ptr(de) if n else None, ptr(tw) if n else None,
                                              ptr(cp) if n else None), "orsp_batch_set_plan")
        self.batch_plan = list(buckets)

    def batch_bbox(self, cost: torch.Tensor, src: torch.Tensor, dst: torch.Tensor, bbox: torch.Tensor,
                   order: Optional[torch.Tensor] = None, delta: Optional[float] = None,
                   path_cap: int = 4096, with_edges: bool = True):
        """K box-ROI searches in one launch.  Returns (nodes[K,cap], edges[K,cap]
        or None, lens[K]) as device tensors; lens < 2 means no path."""
        lib = _lib.load()
        K = int(src.numel())
        if delta is None:
            delta = 0.0  # chosen on the device
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

    def roi_bfs_keep(self, src: int, dst: int, max_depth: int, max_nodes: int, keep) -> torch.Tensor:
        """Bidirectional BFS ROI with extra must-keep nodes (portal seeds).
        Returns roi_nodes (device int32[R])."""
        lib = _lib.load()
        roi = torch.empty(self.N, dtype=torch.int32, device=self.device)
        kp = as_device(np.asarray(keep, dtype=np.int32), torch.int32, self.device)
        cnt = ctypes.c_int32(0)
        check(lib.orsp_roi_bfs_keep(self._h, int(src), int(dst), int(max_depth), int(max_nodes), ptr(kp),
                                    int(kp.numel()), ptr(roi), None, ctypes.byref(cnt), _stream()),
              "orsp_roi_bfs_keep")
        return roi[: cnt.value]

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
        # the ROI extractor whose last result this solver may reuse on the device
        self.roi_source = None
        self._full_roi = None

    def _cost(self, costs) -> torch.Tensor:
        """Device copy of the cost array.  A host array of the drop-in
        accountant (orthoroute_b200.dropin) carries a write counter, so its
        device copy is reused until the host array is written (O(1) per call).
        Any other host array is compared by value with the last one: the
        router calls once per net with the same array, which it also rewrites
        in place between iterations (via pooling, UPF:3381/3443/5298)."""
        if isinstance(costs, torch.Tensor):
            return as_device(costs, torch.float32, self.dg.device)
        mirror = getattr(costs, "_mirror", None)
        if mirror is not None:
            owner, name = mirror
            return owner.device_array(name)
        if hasattr(costs, "__cuda_array_interface__"):  # cupy array from a GPU-mode router
            return as_device(torch.as_tensor(costs, device=self.dg.device), torch.float32, self.dg.device)
        host = np.ascontiguousarray(np.asarray(costs), dtype=np.float32)
        prev_host, prev_dev = self._cost_cache
        if prev_host is not None and prev_host.shape == host.shape and \
                np.array_equal(prev_host.view(np.uint32), host.view(np.uint32)):
            return prev_dev
        t = torch.from_numpy(host).to(self.dg.device)
        self._cost_cache = (host.copy(), t)
        return t

    def _is_full_roi(self, roi_nodes) -> bool:
        """roi_nodes == arange(N) (the reference's full-graph ROI for long nets,
        UPF:4656-4660); checked once per array object."""
        if len(roi_nodes) != self.N or isinstance(roi_nodes, torch.Tensor):
            return False
        if self._full_roi is not None and self._full_roi[0] is roi_nodes:
            return self._full_roi[1]
        a = np.asarray(roi_nodes)
        full = bool(int(a[0]) == 0 and int(a[-1]) == self.N - 1 and
                    np.array_equal(a, np.arange(self.N, dtype=a.dtype)))
        self._full_roi = (roi_nodes, full)
        return full

    def _roi_device(self, roi_nodes, global_to_roi):
        """The ROI node list on the device, or None when global_to_roi is not
        the inverse of roi_nodes (then the caller's map is used as given).
        The check samples positions of the list (both ends, the middle)."""
        if isinstance(roi_nodes, torch.Tensor):
            return as_device(roi_nodes, torch.int32, self.dg.device)
        n = len(roi_nodes)
        if global_to_roi is not None and not isinstance(global_to_roi, torch.Tensor):
            for k in {0, n // 2, n - 1}:
                if int(global_to_roi[int(roi_nodes[k])]) != k:
                    return None
        src = self.roi_source
        if src is not None:
            dev = src.device_roi_for(roi_nodes)
            if dev is not None:
                return dev
        return torch.from_numpy(np.ascontiguousarray(roi_nodes, dtype=np.int32)).to(self.dg.device)

    def find_path_roi_gpu(self, src: int, dst: int, costs, roi_nodes, global_to_roi) -> Optional[List[int]]:
        """CUDADijkstra.find_path_roi_gpu (CD:4909): node path src..dst in global
        ids, or None.  Semantics of SimpleDijkstra.find_path_roi: the search is
        restricted to the ROI and ties between equal distances go to the
        smaller ROI index.  The ROI goes to the device as its node list (O(R)
        per call); global_to_roi is rebuilt there from it."""
        cost = self._cost(costs)
        if len(roi_nodes) == 0:
            return None
        if self._is_full_roi(roi_nodes):
            st, path, _ = self.dg.sssp(cost, int(src), int(dst))
        else:
            roi_d = self._roi_device(roi_nodes, global_to_roi)
            if roi_d is None:
                g2r = as_device(global_to_roi, torch.int32, self.dg.device)
                st, path, _ = self.dg.sssp(cost, int(src), int(dst), roi_map=g2r)
            else:
                st, path = self.dg.sssp_roi_nodes(cost, int(src), int(dst), roi_d)
        if st != _lib.ORSP_OK or path is None or path.numel() < 2:
            return None
        return path.cpu().tolist()

    # SimpleDijkstra.find_path_roi (UPF:1801) has the same signature
    find_path_roi = find_path_roi_gpu

    def find_path_multisource_multisink(self, src_seeds, dst_targets, costs, roi_nodes, global_to_roi):
        """SimpleDijkstra.find_path_multisource_multisink (UPF:1889-1989):
        seeds and targets are [(global node, cost)]; returns (path,
        entry_layer, exit_layer) or None.  Repeated targets keep their last
        cost, as the reference's dict does."""
        cost = self._cost(costs)
        g2r = as_device(global_to_roi, torch.int32, self.dg.device)
        seeds = [int(n) for n, _ in src_seeds]
        scost = np.asarray([float(c) for _, c in src_seeds], dtype=np.float32)
        tmap = {}
        for n, c in dst_targets:
            tmap[int(n)] = float(c)
        if not seeds or not tmap:
            return None
        st, path, _ = self.dg.sssp_multi(cost, seeds, list(tmap.keys()), seed_cost=scost,
                                         target_cost=np.asarray(list(tmap.values()), dtype=np.float64), roi_map=g2r)
        if st != _lib.ORSP_OK or path is None or path.numel() < 2:
            return None
        p = path.cpu().tolist()
        plane = self.dg.nx * self.dg.ny if self.dg.nx > 0 else 0
        if plane:
            return p, p[0] // plane, p[-1] // plane
        return p, 0, 0

    def find_path_fullgraph_gpu_seeds(self, costs, src_seeds, dst_targets, ub_hint=None, *, allowed_bitmap=None,
                                      use_bitmap=False):
        """CUDADijkstra.find_path_fullgraph_gpu_seeds (CD:5467): path from the
        best seed to the best target over the whole graph (restricted to the
        allowed bitmap when use_bitmap), or None.  Exact shortest path; the
        reference wavefront instead stops at the first target it reaches."""
        if len(src_seeds) == 0 or len(dst_targets) == 0:
            return None
        cost = self._cost(costs)
        roi = None
        if use_bitmap and allowed_bitmap is not None:
            bm = allowed_bitmap.get() if hasattr(allowed_bitmap, "get") else allowed_bitmap
            roi = self.dg.roi_from_bitmap(np.asarray(bm).view(np.int32))
        targets = np.unique(np.asarray(dst_targets, dtype=np.int32))
        st, path, _ = self.dg.sssp_multi(cost, np.asarray(src_seeds, dtype=np.int32), targets, roi_map=roi)
        if st != _lib.ORSP_OK or path is None or path.numel() < 2:
            return None
        return path.cpu().tolist()

    def find_paths_on_rois(self, roi_batch, use_bitmap: bool = True):
        """CUDADijkstra.find_paths_on_rois (CD:2014-2086): K ROI subgraphs given
        as 13-tuples (src, dst, indptr, indices, weights, roi_size, bitmap,
        bbox x 6) in ROI-local ids (CD:55-91).  Returns one path (local ids)
        or None per ROI.  The local CSRs are concatenated into one graph and
        searched in one launch with node-range ROIs; with use_bitmap a node
        whose bit is clear is never entered (edges into it are +inf), as the
        reference's IN_BITMAP check does (CD:237-239)."""
        K = len(roi_batch)
        if K == 0:
            return []
        node_off = [0]
        edge_off = [0]
        for t in roi_batch:
            node_off.append(node_off[-1] + int(len(t[2]) - 1))
            edge_off.append(edge_off[-1] + int(len(t[3])))
        Ntot, Etot = node_off[-1], edge_off[-1]
        indptr = np.empty(Ntot + 1, dtype=np.int64)
        indices = np.empty(Etot, dtype=np.int32)
        weights = np.empty(Etot, dtype=np.float32)
        src = np.empty(K, dtype=np.int32)
        dst = np.empty(K, dtype=np.int32)
        ranges = np.empty((K, 2), dtype=np.int32)
        for k, t in enumerate(roi_batch):
            s_, d_, ip, ix, w = t[0], t[1], t[2], t[3], t[4]
            ip = (ip.get() if hasattr(ip, "get") else np.asarray(ip)).astype(np.int64)
            ix = (ix.get() if hasattr(ix, "get") else np.asarray(ix)).astype(np.int64)
            w = (w.get() if hasattr(w, "get") else np.asarray(w)).astype(np.float32).copy()
            n0, e0 = node_off[k], edge_off[k]
            n = node_off[k + 1] - n0
            bm = t[6] if len(t) > 6 else None
            if use_bitmap and bm is not None:
                bm = (bm.get() if hasattr(bm, "get") else np.asarray(bm)).astype(np.uint32).reshape(-1)
                word = ix >> 5
                ok = (word < len(bm)) & (((bm[np.minimum(word, len(bm) - 1)] >> (ix & 31).astype(np.uint32)) & 1) == 1)
                w[~ok] = np.float32(np.inf)
            indptr[n0: n0 + n + 1] = ip + e0
            indices[e0: e0 + len(ix)] = ix + n0
            weights[e0: e0 + len(ix)] = w
            src[k] = int(s_) + n0
            dst[k] = int(d_) + n0
            ranges[k] = (n0, n0 + n)
        if Etot >= 2 ** 31 or Ntot >= 2 ** 31:
            raise ValueError("ROI batch too large for int32 ids")
        dg = DeviceGraph(indptr.astype(np.int32), indices, device=self.dg.device)
        wt = torch.from_numpy(weights).to(self.dg.device)
        cap = int(max(n1 - n0 for n0, n1 in ranges) + 1)
        lib = _load_lib()
        nodes = torch.empty((K, cap), dtype=torch.int32, device=self.dg.device)
        lens = torch.zeros(K, dtype=torch.int32, device=self.dg.device)
        # keep the device copies referenced until the launch has been issued
        src_d = torch.from_numpy(src).to(self.dg.device)
        dst_d = torch.from_numpy(dst).to(self.dg.device)
        ranges_d = torch.from_numpy(ranges).to(self.dg.device)
        check(lib.orsp_sssp_batch_ranges(dg.handle, ptr(wt), K, ptr(src_d), ptr(dst_d), ptr(ranges_d), None,
                                         0.0, ptr(nodes), None, cap, ptr(lens),
                                         _stream()), "orsp_sssp_batch_ranges")
        lens_h = lens.cpu().numpy()
        nodes_h = nodes.cpu().numpy()
        out = []
        for k in range(K):
            L = int(lens_h[k])
            out.append((nodes_h[k, :L] - node_off[k]).tolist() if L >= 2 else None)
        dg.close()
        return out

    def path_to_edges_list(self, node_path) -> list:
        """PathFinderRouter._path_to_edges (UPF:5463-5476) on the device: the
        first CSR edge u->v for each consecutive pair, pairs without an edge
        skipped; returns a Python list like the reference."""
        if len(node_path) < 2:
            return []
        p = torch.as_tensor(np.asarray(node_path, dtype=np.int32)).to(self.dg.device)
        return self.dg.path_to_edges(p).cpu().tolist()
