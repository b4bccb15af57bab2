"""The whole B200 drop-in for an unmodified OrthoRoute PathFinderRouter.

The reference's negotiation loop (orthoroute/algorithms/manhattan/
unified_pathfinder.py, PathFinderRouter._pathfinder_negotiation UPF:3548-4259
and _route_all UPF:4441-4823) reaches the hot path through four hooks
(EdgeAccountant, ROIExtractor, SimpleDijkstra and _path_to_edges) plus two
router methods that rewrite the cost array (_apply_via_pooling_penalties
UPF:3243-3387, _block_via_edges_with_collisions UPF:3448-3546).  ``install``
replaces all of them with objects that run on the GPU; net order, rip-up and
the loop itself stay the reference's.

The reference loop also reads and writes the accountant's arrays directly
with numpy (``present.fill(0)``, ``pres[idx] += penalty``,
``accounting.present_ema = accounting.present.copy()``, UPF:3651, 3868,
4977-4985), and with its ``use_gpu`` flag clear it treats them as host
arrays.  So the accountant here keeps every array twice: a host array that
the reference sees (pinned memory, so copies are fast) and a device copy that
the kernels use.  The host array counts its writes (``TrackedArray``); a
device copy is refreshed only when its host array was written since, and the
result of every device update is copied back to the host array.  The per-net
cost array the searches read (``total_cost``) therefore crosses to the device
once per iteration, not once per net.
"""
from __future__ import annotations

from collections import Counter
from types import MethodType
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .solver import DeviceGraph, GpuSolver, _require_cuda, _stream, as_device


# ----------------------------------------------------------------------------
class TrackedArray(np.ndarray):
    """A host array that counts writes made through numpy: item and slice
    assignment, ``fill``, in-place operators and ufuncs with ``out=`` or
    ``.at``.  Views share the counter of the array they view.  Arithmetic on
    it returns plain ndarrays."""

    def __new__(cls, arr):
        obj = np.asarray(arr).view(cls)
        obj._ver = [0]
        return obj

    def __array_finalize__(self, obj):
        ver = getattr(obj, "_ver", None)
        self._ver = ver if ver is not None else [0]

    @property
    def version(self) -> int:
        return self._ver[0]

    def __setitem__(self, key, value):
        np.ndarray.__setitem__(self.view(np.ndarray), key, value)
        self._ver[0] += 1

    def fill(self, value):
        self.view(np.ndarray).fill(value)
        self._ver[0] += 1

    def __array_ufunc__(self, ufunc, method, *inputs, out=None, **kwargs):
        args = [x.view(np.ndarray) if isinstance(x, TrackedArray) else x for x in inputs]
        if out is not None:
            kwargs["out"] = tuple(o.view(np.ndarray) if isinstance(o, TrackedArray) else o for o in out)
        res = getattr(ufunc, method)(*args, **kwargs)
        if method == "at" and isinstance(inputs[0], TrackedArray):
            inputs[0]._ver[0] += 1
        if out is not None:
            for o in out:
                if isinstance(o, TrackedArray):
                    o._ver[0] += 1
            return out[0] if len(out) == 1 else out
        return res


def _pinned_host(n: int, fill: float) -> TrackedArray:
    buf = torch.empty(n, dtype=torch.float32).pin_memory().numpy()
    buf.fill(fill)
    return TrackedArray(buf)


def _f32(x: float) -> float:
    """Python float -> the float32 value numpy uses for a weak scalar."""
    return float(np.float32(x))


class _ConstCache:
    """Device copies of host arrays the caller passes again and again
    (base costs, edge layers, edge kinds): re-uploaded only when the values
    change (one host comparison per call, the calls are per iteration)."""

    def __init__(self, device):
        self.device = device
        self._c = {}

    def get(self, key, arr, dtype):
        if arr is None:
            return None
        if isinstance(arr, torch.Tensor):
            return as_device(arr, dtype, self.device)
        host = np.asarray(arr)
        hit = self._c.get(key)
        if hit is not None and hit[0].shape == host.shape and hit[0].dtype == host.dtype and \
                np.array_equal(hit[0], host):
            return hit[1]
        dev = as_device(host, dtype, self.device)
        self._c[key] = (host.copy(), dev)
        return dev


# ----------------------------------------------------------------------------
class MirroredEdgeAccountant:
    """``router.accounting``: the EdgeAccountant interface (UPF:799-1068) with
    host arrays for the reference loop and the arithmetic on the GPU.

    ``present``, ``present_ema``, ``history``, ``capacity``, ``total_cost``
    are float32 ``TrackedArray`` host arrays; ``canonical`` is the same dict
    the reference keeps.  ``use_gpu`` is False because that flag selects the
    reference's host-array branches (``.get()`` / ``cp.asarray`` otherwise);
    the per-iteration O(E) updates (costs, history, EMA, overuse) run on the
    device all the same."""

    ARRAYS = ("present", "present_ema", "history", "capacity", "total_cost")

    def __init__(self, num_edges: int, device=None):
        _require_cuda()
        object.__setattr__(self, "_host", {})
        self.E = int(num_edges)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.canonical = {}
        self.use_gpu = False
        self.xp = np
        self._dev = {}
        self._synced = {}
        for name in self.ARRAYS:
            if name == "total_cost":
                self._host[name] = None  # set by the first update_costs, as the reference does
                continue
            self._new_array(name, 1.0 if name == "capacity" else 0.0)
        self._consts = _ConstCache(self.device)
        self._over2 = torch.zeros(2, dtype=torch.int64, device=self.device)
        self._over2_h = torch.zeros(2, dtype=torch.int64).pin_memory()

    @classmethod
    def replacing(cls, old, device=None) -> "MirroredEdgeAccountant":
        """A mirrored accountant holding the state of `old` (a reference
        EdgeAccountant, possibly mid-run)."""
        acct = cls(int(old.E), device=device)
        acct.canonical = dict(getattr(old, "canonical", {}))
        for name in cls.ARRAYS:
            v = getattr(old, name, None)
            if v is not None:
                setattr(acct, name, v.get() if hasattr(v, "get") else v)
        return acct

    # --- host / device mirrors ----------------------------------------------
    def _new_array(self, name: str, fill: float):
        h = _pinned_host(self.E, fill)
        h._mirror = (self, name)
        self._host[name] = h
        self._dev[name] = torch.full((self.E,), fill, dtype=torch.float32, device=self.device)
        self._synced[name] = h.version

    def __getattr__(self, name):
        host = object.__getattribute__(self, "_host")
        if name in host:
            return host[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in MirroredEdgeAccountant.ARRAYS:
            self._assign(name, value)
        else:
            object.__setattr__(self, name, value)

    def _assign(self, name: str, value):
        """Rebinding an array (the reference does ``present_ema =
        present.copy()``) copies the values into this accountant's buffer."""
        if value is None:
            self._host[name] = None
            return
        cur = self._host.get(name)
        if value is cur:
            cur._ver[0] += 1
            return
        arr = value.detach().cpu().numpy() if isinstance(value, torch.Tensor) else np.asarray(value)
        if arr.shape != (self.E,):
            raise ValueError(f"accounting.{name} must have {self.E} entries, got shape {arr.shape}")
        if cur is None:
            self._new_array(name, 0.0)
            cur = self._host[name]
        np.copyto(cur.view(np.ndarray), arr, casting="same_kind")
        cur._ver[0] += 1

    def device_array(self, name: str) -> torch.Tensor:
        """The device copy of a host array, uploaded first if the host array
        was written since the last upload or download."""
        h = self._host[name]
        d = self._dev[name]
        if self._synced[name] != h.version:
            d.copy_(torch.from_numpy(h.view(np.ndarray)), non_blocking=True)
            self._synced[name] = h.version
        return d

    def _pull(self, name: str):
        """Device result -> host array (the write does not count as a host
        write: the two copies are equal afterwards)."""
        h = self._host[name]
        torch.from_numpy(h.view(np.ndarray)).copy_(self._dev[name])
        self._synced[name] = h.version

    # --- canonical store (host, as the reference's dict) ---------------------
    def refresh_from_canonical(self):
        """present = float(count) from the canonical dict (UPF:814-819)."""
        p = self.present
        p.fill(0)
        if self.canonical:
            k = np.fromiter(self.canonical.keys(), dtype=np.int64, count=len(self.canonical))
            v = np.fromiter(self.canonical.values(), dtype=np.float64, count=len(self.canonical))
            ok = (k >= 0) & (k < self.E)
            p[k[ok]] = v[ok].astype(np.float32)

    def commit_path(self, edge_indices):
        """count += 1 and present += 1 per edge, repeats included (UPF:821-826)."""
        idx = [int(i) for i in edge_indices]
        if not idx:
            return
        c = self.canonical
        for i in idx:
            c[i] = c.get(i, 0) + 1
        np.add.at(self.present, np.asarray(idx, dtype=np.int64), np.float32(1))

    def clear_path(self, edge_indices):
        """count -= 1 (entries at 0 removed) and present = max(0, present - 1)
        per edge (UPF:828-836).  Subtracting 1 from a float32 below 2^24 is
        exact, so subtracting each edge's repeat count at once and clamping
        gives the bits of the reference's one-by-one loop."""
        idx = [int(i) for i in edge_indices]
        if not idx:
            return
        c = self.canonical
        for i in idx:
            if i in c:
                c[i] -= 1
                if c[i] <= 0:
                    del c[i]
        cnt = Counter(idx)
        k = np.fromiter(cnt.keys(), dtype=np.int64, count=len(cnt))
        n = np.fromiter(cnt.values(), dtype=np.float32, count=len(cnt))
        p = self.present
        p[k] = np.maximum(np.float32(0), p.view(np.ndarray)[k] - n)

    def verify_present_matches_canonical(self) -> bool:
        """UPF:878-896."""
        rec = np.zeros(self.E, dtype=np.float32)
        for i, cnt in self.canonical.items():
            if 0 <= i < self.E:
                rec[i] = float(cnt)
        return bool(np.sum(np.abs(self.present.view(np.ndarray) - rec)) <= 0.01)

    # --- per-iteration updates on the device --------------------------------
    def compute_overuse(self, router_instance=None):
        """(edge overuse sum + via column/segment overuse, overused edge count)
        (UPF:838-876); the edge part on the device."""
        lib = _lib.load()
        check(lib.orsp_overuse(self.E, ptr(self.device_array("present")), ptr(self.device_array("capacity")),
                               ptr(self._over2), ptr(self._over2_h), _stream()), "orsp_overuse")
        s, c = (int(v) for v in self._over2_h.tolist())
        if router_instance is not None:
            for use, cap in (("via_col_use", "via_col_cap"), ("via_seg_use", "via_seg_cap")):
                if hasattr(router_instance, use) and hasattr(router_instance, cap):
                    u = np.asarray(getattr(router_instance, use))
                    k = np.asarray(getattr(router_instance, cap))
                    s += int(np.maximum(0, u - k).sum())
        return s, c

    def update_present_ema(self, beta: float = 0.60):
        """present_ema = beta*present + (1-beta)*present_ema (UPF:963-971)."""
        check(_lib.load().orsp_update_present_ema(self.E, ptr(self.device_array("present")),
                                                  ptr(self.device_array("present_ema")), _f32(beta),
                                                  _f32(1.0 - beta), _stream()), "orsp_update_present_ema")
        self._pull("present_ema")

    def update_history(self, gain: float, base_costs=None, history_cap_multiplier: float = 10.0,
                       decay_factor: float = 0.98, use_raw_present: bool = False):
        """UPF:898-961."""
        base = self._consts.get("base", base_costs, torch.float32)
        pres = self.device_array("present" if use_raw_present else "present_ema")
        check(_lib.load().orsp_update_history(self.E, ptr(self.device_array("history")), ptr(pres),
                                              ptr(self.device_array("capacity")), ptr(base), _f32(gain),
                                              _f32(history_cap_multiplier), _f32(decay_factor), _stream()),
              "orsp_update_history")
        self._pull("history")

    def update_costs(self, base_costs, pres_fac: float, hist_weight: float = 1.0, add_jitter: bool = True,
                     via_cost_multiplier: float = 1.0, base_cost_weight: float = 0.01, *, edge_layer=None,
                     layer_bias_per_layer=None, edge_kind=None):
        """UPF:973-1043, into ``total_cost``."""
        base = self._consts.get("base", base_costs, torch.float32)
        use_bias = edge_layer is not None and layer_bias_per_layer is not None and edge_kind is not None
        el = self._consts.get("edge_layer", edge_layer, torch.uint8) if use_bias else None
        ek = self._consts.get("edge_kind", edge_kind, torch.uint8) if use_bias else None
        lb = as_device(np.asarray(layer_bias_per_layer, dtype=np.float32), torch.float32,
                       self.device) if use_bias else None
        if self._host.get("total_cost") is None:
            self._new_array("total_cost", 0.0)
        check(_lib.load().orsp_update_costs(self.E, ptr(base), ptr(self.device_array("present_ema")),
                                            ptr(self.device_array("capacity")), ptr(self.device_array("history")),
                                            ptr(el), ptr(ek), ptr(lb), _f32(pres_fac), _f32(hist_weight),
                                            _f32(via_cost_multiplier), _f32(base_cost_weight),
                                            1 if add_jitter else 0, ptr(self._dev["total_cost"]), _stream()),
              "orsp_update_costs")
        self._pull("total_cost")


# ----------------------------------------------------------------------------
class DropInROIExtractor:
    """``router.roi_extractor``: ROIExtractor.extract_roi / extract_roi_bfs
    (UPF:1619-1734) on the GPU, portal seeds included.  Returns host arrays
    like the reference; the device copy of the last ROI stays available to
    the solver, which then needs no upload."""

    def __init__(self, dg: DeviceGraph, lattice=None, max_roi_nodes: int = 50_000):
        self.dg = dg
        self.N = dg.N
        self.lattice = lattice
        self.max_roi_nodes = int(max_roi_nodes)
        self._last = None  # (host roi array, device roi tensor)

    def _xy(self, n: int):
        lat = self.lattice
        if hasattr(lat, "idx_to_coord"):  # the reference's Lattice3D
            x, y, _ = lat.idx_to_coord(int(n))
        else:
            x, y, _ = lat.coords(int(n))
        return int(x), int(y)

    def extract_roi(self, src: int, dst: int, initial_radius: int = 40, stagnation_bonus: float = 0.0,
                    portal_seeds: list = None):
        """UPF:1619-1634: radius = max(60, int(0.75*manhattan + 2*bonus)) on a lattice."""
        if self.lattice is not None:
            sx, sy = self._xy(src)
            dx, dy = self._xy(dst)
            manhattan = abs(dx - sx) + abs(dy - sy)
            radius = max(60, int(manhattan * 0.75 + stagnation_bonus * 2.0))
        else:
            radius = initial_radius
        return self.extract_roi_bfs(src, dst, initial_radius=radius, stagnation_bonus=stagnation_bonus,
                                    portal_seeds=portal_seeds)

    def extract_roi_bfs(self, src: int, dst: int, initial_radius: int = 40, stagnation_bonus: float = 0.0,
                        portal_seeds: list = None):
        """UPF:1636-1734: bidirectional BFS to depth min(radius + 2*bonus, 150),
        portal seeds kept as must-keep nodes, at most max_roi_nodes nodes."""
        max_depth = min(int(initial_radius + stagnation_bonus * 2.0), 150)
        keep = [int(n) for n, _ in portal_seeds] if portal_seeds else []
        roi_d = self.dg.roi_bfs_keep(int(src), int(dst), max_depth, self.max_roi_nodes, keep)
        roi = roi_d.cpu().numpy()
        g2r = np.full(self.N, -1, dtype=np.int32)
        g2r[roi] = np.arange(len(roi), dtype=np.int32)
        self._last = (roi, roi_d)
        return roi, g2r

    def device_roi_for(self, roi_nodes) -> Optional[torch.Tensor]:
        """The device copy of `roi_nodes` if it is the last ROI returned."""
        if self._last is not None and self._last[0] is roi_nodes:
            return self._last[1]
        return None


# ----------------------------------------------------------------------------
def _device_via_penalties(router, acct: MirroredEdgeAccountant, dg: DeviceGraph, original):
    """_apply_via_pooling_penalties (UPF:3243-3387) on the device: the
    vectorised branch the reference takes when its via metadata exists (the
    metadata-less case keeps the reference's sequential fallback)."""

    def apply(pres_fac: float):
        if not hasattr(router, "via_col_pres") and not hasattr(router, "via_seg_pres"):
            return None
        if getattr(router, "_via_edge_metadata", None) is None or acct.total_cost is None:
            return original(pres_fac)
        cfg = router.config
        col_w = _f32(float(getattr(cfg, "via_column_weight", 1.0)))
        seg_w = _f32(float(getattr(cfg, "via_segment_weight", 1.0)))
        dev = acct.device
        col = getattr(router, "via_col_pres", None)
        pre = getattr(router, "via_seg_prefix", None)
        col_d = None if col is None else as_device(np.ascontiguousarray(col, dtype=np.float32).reshape(-1),
                                                   torch.float32, dev)
        pre_d = None if pre is None else as_device(np.ascontiguousarray(pre, dtype=np.float32).reshape(-1),
                                                   torch.float32, dev)
        lb_d, f64, k = None, 0, 0.0
        if hasattr(router, "layer_bias"):
            lb = np.asarray(router.layer_bias)
            f64 = 1 if lb.dtype == np.float64 else 0
            lb_d = as_device(lb.astype(np.float64), torch.float64, dev)
            k = float(getattr(cfg, "via_hot_layer_discount", 0.20))
        check(_lib.load().orsp_via_penalties(dg.handle, ptr(col_d), ptr(pre_d), ptr(lb_d), f64, k, col_w, seg_w,
                                             _f32(pres_fac), ptr(acct.device_array("total_cost")), _stream()),
              "orsp_via_penalties")
        acct._pull("total_cost")
        return None

    return apply


def _device_hard_block(router, acct: MirroredEdgeAccountant, dg: DeviceGraph):
    """_block_via_edges_with_collisions (UPF:3448-3546) on the device: via
    edges whose column, or any segment they span, is at capacity become +inf."""

    def block():
        if getattr(router, "_via_edge_metadata", None) is None:
            return None
        if not hasattr(router, "via_col_use") and not hasattr(router, "via_seg_use"):
            return None
        if acct.total_cost is None:
            return None
        dev = acct.device

        def i32(name):
            a = getattr(router, name, None)
            return None if a is None else as_device(np.ascontiguousarray(a, dtype=np.int32).reshape(-1),
                                                    torch.int32, dev)

        cu, cc, su, sc = i32("via_col_use"), i32("via_col_cap"), i32("via_seg_use"), i32("via_seg_cap")
        if cu is None or cc is None:
            cu = cc = None
        if su is None or sc is None:
            su = sc = None
        check(_lib.load().orsp_via_hard_block(dg.handle, ptr(cu), ptr(cc), ptr(su), ptr(sc),
                                              ptr(acct.device_array("total_cost")), _stream()),
              "orsp_via_hard_block")
        acct._pull("total_cost")
        return None

    return block


class DropInSet:
    """The drop-in objects for one graph, without a router: the mirrored
    accountant, the ROI extractor, the solver, path -> edges and the two via
    steps (which read the router state they need from the object passed to
    them).  ``install`` wires the same objects into a router; this class
    serves callers that drive their own loop (and the recorded-run replay)."""

    def __init__(self, indptr, indices, lattice=None, nx: int = 0, ny: int = 0, nz: int = 0, device=None,
                 max_roi_nodes: int = 50_000):
        _require_cuda()
        self.dg = DeviceGraph(indptr, indices, nx, ny, nz, device=device)
        self.acct = MirroredEdgeAccountant(self.dg.E, device=self.dg.device)
        self.extractor = DropInROIExtractor(self.dg, lattice, max_roi_nodes=max_roi_nodes)
        self.solver = GpuSolver(self.dg, lattice)
        self.solver.roi_source = self.extractor

    def extract_roi(self, src, dst, initial_radius=40, stagnation_bonus=0.0, portal_seeds=None):
        return self.extractor.extract_roi(src, dst, initial_radius, stagnation_bonus, portal_seeds)

    def find_path_roi(self, src, dst, costs, roi_nodes, global_to_roi):
        return self.solver.find_path_roi(src, dst, costs, roi_nodes, global_to_roi)

    def path_to_edges(self, path):
        return self.solver.path_to_edges_list(path)

    def via_penalties(self, router_state, pres_fac):
        def original(_):
            raise RuntimeError("via penalties without via metadata are not handled on the device")
        return _device_via_penalties(router_state, self.acct, self.dg, original)(pres_fac)

    def via_block(self, router_state):
        return _device_hard_block(router_state, self.acct, self.dg)()


def install(router, *, device=None, accounting: bool = True, roi: bool = True, via: bool = True,
            path_to_edges: bool = True):
    """Wires the whole B200 path into an initialised router (after
    ``router.initialize_graph``).  Returns the GpuSolver.

    - ``router.solver.find_path_roi`` / ``find_path_multisource_multisink``
      (SimpleDijkstra, UPF:1801-1989) become the GPU searches.  The
      ``gpu_solver`` slot is left as it is: with portals, ``_route_all``
      imports CuPy inside the try block of its GPU fast path (UPF:4536-4603)
      and marks the net failed when that import fails, so a CuPy-free
      process must not take that branch.
    - ``router.accounting`` becomes a MirroredEdgeAccountant holding the
      current state; ``router.roi_extractor`` a DropInROIExtractor;
      ``router._path_to_edges`` the device mapping; the via pooling penalty
      and the via hard block run on the device.
    Nothing falls back to the CPU: every hook raises if the CUDA library is
    missing."""
    if getattr(router, "graph", None) is None or getattr(router, "solver", None) is None:
        raise RuntimeError("install() needs an initialised router (call initialize_graph first)")
    _require_cuda()
    g = router.graph
    lat = router.lattice
    indptr = g.indptr.get() if hasattr(g.indptr, "get") else np.asarray(g.indptr)
    indices = g.indices.get() if hasattr(g.indices, "get") else np.asarray(g.indices)
    nx = getattr(lat, "x_steps", 0) if lat is not None else 0
    ny = getattr(lat, "y_steps", 0) if lat is not None else 0
    nz = getattr(lat, "layers", 0) if lat is not None else 0
    dg = DeviceGraph(indptr, indices, nx, ny, nz, device=device)
    solver = GpuSolver(dg, lat)
    s = router.solver
    s.find_path_roi = solver.find_path_roi
    s.find_path_multisource_multisink = solver.find_path_multisource_multisink
    if accounting:
        acct = MirroredEdgeAccountant.replacing(router.accounting, device=dg.device)
        router.accounting = acct
    if roi:
        old = getattr(router, "roi_extractor", None)
        ex = DropInROIExtractor(dg, lat, max_roi_nodes=getattr(old, "max_roi_nodes", 50_000))
        router.roi_extractor = ex
        solver.roi_source = ex
    if via and accounting:
        router._apply_via_pooling_penalties = _device_via_penalties(router, router.accounting, dg,
                                                                    router._apply_via_pooling_penalties)
        router._block_via_edges_with_collisions = _device_hard_block(router, router.accounting, dg)
    if path_to_edges:
        router._path_to_edges = solver.path_to_edges_list
    router._orsp_solver = solver
    return solver
