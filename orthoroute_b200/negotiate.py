"""PathFinder negotiated-congestion routing on the device kernels.

This is the loop of PathFinderRouter._pathfinder_negotiation
(orthoroute/algorithms/manhattan/unified_pathfinder.py:3548-4259, "UPF") and
_route_all (UPF:4441-4823) reduced to the plain PathFinder schedule the
benchmark configurations name, with every array step on the GPU:

  per iteration
    present <- committed usage                         refresh_from_canonical  UPF:814
    present_ema <- present (iteration 1), then EMA     update_present_ema      UPF:963, 3648-3654
    total_cost <- base/present/history formula         update_costs            UPF:973, 3725
    route the nets (rip up the old path, ROI, SSSP,    _route_all              UPF:4441
      backtrace, path -> edges, commit)
    present <- usage; overuse count                    compute_overuse         UPF:838, 3880
    stop at zero overuse with every net routed         UPF:4023-4027, 4121
    history update (raw present, cap 15*base,          update_history          UPF:898, 4030-4057
      decay 0.98 from iteration 10, gain x1.25 <= 1.2 from iteration 8)
    pres_fac <- min(pres_fac * mult, pres_fac_max)     UPF:4224

Costs are computed once per iteration and are read-only while the nets are
routed (UPF:4459, "Sequential routing with FIXED costs throughout
iteration"), so each net's search depends only on that iteration's costs and
its own ROI.  Two execution modes therefore give identical paths:

* ``mode="sequential"``: one persistent grid search per net (the plain GPU
  path, a host round trip per net);
* ``mode="batched"``: every net of the iteration in one launch of the
  batched box-ROI kernel, then one batched commit.

Heuristics of the reference loop that are not part of plain PathFinder (layer
bias, via pooling, hotset sampling with random.seed, barrel-conflict
penalties, stagnation rip-up) are not applied here; the accounting entry
points for them exist in the library and are exercised by the tests.

Cost policies (``NegotiationConfig.cost_update``):

* ``"iteration"`` - the reference's: present_ema-based costs computed once per
  iteration (above).  On the benchmark lattice this schedule oscillates and
  does not reach zero overuse (neither does the reference's own loop).
* ``"net"`` - classic PathFinder, the per-net refresh the reference's
  EdgeAccountant.update_present_cost_only (UPF:1045-1068) is meant for: after
  each net is ripped up or committed, the costs of the edges it touched are
  recomputed from live usage, ``base*w + pres_fac*max(0, usage+1-cap) +
  hist_w*history + jitter``, so every net sees the nets routed before it.  A
  net's search reads only costs inside its box and its rip-up / commit touch
  only edges inside its box, so nets whose boxes are pairwise disjoint see
  exactly the sequential costs: batched mode launches one "level" of such
  nets at a time (level(j) = 1 + max level of the earlier nets whose box
  intersects j's), giving the sequential result bit for bit.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .accounting import DeviceEdgeAccountant
from .lattice import Lattice, bbox_with_margin
from .roi import DeviceROIExtractor
from .solver import DeviceGraph, _stream, as_device


@dataclass
class NegotiationConfig:
    max_iterations: int = 30
    pres_fac_init: float = 0.5
    pres_fac_mult: float = 1.5
    pres_fac_max: float = 64.0
    hist_gain: float = 1.0
    hist_gain_boost: bool = True
    hist_cost_weight: float = 1.0
    base_cost_weight: float = 1.0
    via_cost_multiplier: float = 1.0
    present_ema_beta: float = 0.4
    history_cap_multiplier: float = 15.0
    history_decay: float = 0.98
    history_decay_from: int = 10
    add_jitter: bool = True
    roi: str = "bbox"  # "bbox" | "bfs" | "full"
    roi_margin: int = 10
    reroute: str = "all"  # "all" | "offenders"
    full_graph_retry: bool = True
    delta: Optional[float] = None
    path_cap: int = 4096
    cost_update: str = "iteration"  # "iteration" (reference) | "net" (live usage)
    native_loop: bool = True  # per-net policy on a lattice: orsp_route_nets (no host round trip per net)
    net_order: str = "index"  # "index" | "disjoint": first-fit rounds of pairwise disjoint boxes
    stall_grow: int = 0  # cells added to the margin of a net that offends stall_iterations times running
    stall_iterations: int = 2
    first_pass: str = "sequential"  # per-net costs: "sequential", or "independent" (iteration 1 on fixed costs)
    batch_plan: Optional[list] = None  # DeviceGraph.set_batch_plan for the batched searches
    # per-net costs, batched mode: 0 = each net sees every earlier net (one
    # launch per round of disjoint boxes); G > 0 = snapshot groups of G
    # consecutive nets of the order, searched together on the costs after the
    # group's rip-ups and then committed together (the nets of a group do not
    # see one another)
    group_nets: int = 0
    group_repair: int = 0  # snapshot groups: rounds of re-search for nets sharing an edge with an earlier group-mate


@dataclass
class IterationStats:
    iteration: int
    pres_fac: float
    routed: int
    failed: int
    over_sum: int
    over_cnt: int
    nets_searched: int
    seconds: float


@dataclass
class RouteResult:
    converged: bool
    iterations: List[IterationStats]
    seconds: float
    paths: List[np.ndarray]
    edge_usage: np.ndarray
    wirelength: int
    vias: int
    meta: dict = field(default_factory=dict)

    def overuse_trace(self):
        return [(s.over_sum, s.over_cnt) for s in self.iterations]


def level_schedule(boxes: np.ndarray) -> np.ndarray:
    """level[j] = 1 + max(level[i] for i < j whose box intersects box j), 0
    when none does; nets of one level have pairwise disjoint boxes and each
    follows every earlier net it overlaps."""
    M = len(boxes)
    lv = np.zeros(M, dtype=np.int32)
    if M == 0:
        return lv
    x0, x1, y0, y1, z0, z1 = (boxes[:, i] for i in range(6))
    for j in range(1, M):
        inter = ((x0[:j] <= x1[j]) & (x1[:j] >= x0[j]) & (y0[:j] <= y1[j]) & (y1[:j] >= y0[j])
                 & (z0[:j] <= z1[j]) & (z1[:j] >= z0[j]))
        if inter.any():
            lv[j] = int(lv[:j][inter].max()) + 1
    return lv


GROUP_MAX = 1024  # nets per device launch (orsp_route_nets group limit)


def level_groups(idx: np.ndarray, lv: np.ndarray, group_max: int = GROUP_MAX):
    """Order and group_ptr for orsp_route_nets: the nets of each level in their
    original order, level after level, each level cut into chunks of at most
    group_max nets.  Every net still follows each earlier net whose box meets
    its own, so the result equals routing `idx` one net at a time."""
    order = []
    ptr_ = [0]
    for L in range(int(lv.max()) + 1 if len(lv) else 0):
        sel = idx[lv == L]
        for a in range(0, len(sel), group_max):
            chunk = sel[a:a + group_max]
            order.append(chunk)
            ptr_.append(ptr_[-1] + len(chunk))
    order = np.concatenate(order).astype(np.int32) if order else np.zeros(0, np.int32)
    return order, np.asarray(ptr_, dtype=np.int32)


def disjoint_order(boxes: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Nets of idx reordered into first-fit rounds: each net joins the first
    round whose boxes it does not meet; rounds are concatenated.  Under this
    order the level schedule of the nets is exactly the rounds, so one launch
    per round gives the one-net-at-a-time result of the same order."""
    idx = np.asarray(idx)
    if idx.size == 0:
        return idx
    b = boxes[idx]
    rnd = np.full(idx.size, -1, dtype=np.int64)
    nrounds = 0
    for j in range(idx.size):
        r = 0
        if j:
            p = b[:j]
            meet = ((p[:, 0] <= b[j, 1]) & (b[j, 0] <= p[:, 1]) & (p[:, 2] <= b[j, 3]) & (b[j, 2] <= p[:, 3])
                    & (p[:, 4] <= b[j, 5]) & (b[j, 4] <= p[:, 5]))
            taken = np.zeros(nrounds + 1, dtype=bool)
            taken[rnd[:j][meet]] = True
            r = int(np.argmin(taken))
        rnd[j] = r
        nrounds = max(nrounds, r + 1)
    return idx[np.argsort(rnd, kind="stable")]


class PathFinder:
    def __init__(self, lattice: Lattice, base_cost=None, config: Optional[NegotiationConfig] = None, device=None):
        self.lat = lattice
        self.cfg = config or NegotiationConfig()
        self.dg = DeviceGraph.from_lattice(lattice, device=device)
        self.device = self.dg.device
        self.E = lattice.E
        base = lattice.base_cost if base_cost is None else base_cost
        self.base = as_device(base, torch.float32, self.device)
        self.edge_kind = np.asarray(lattice.edge_kind)
        self.roi = DeviceROIExtractor(self.dg, lattice=lattice, return_device=True)
        self._owner = None
        self._searches = 0

    # ------------------------------------------------------------------
    def _offenders(self, acc, net_edges, net_lens, nets_all):
        over = (acc.present > acc.capacity)
        cap = net_edges.shape[1]
        # only the first len-1 entries of a row are edges of the net's path
        valid = torch.arange(cap, device=self.device)[None, :] < (net_lens.long() - 1).clamp_min(0)[:, None]
        e = torch.where(valid, net_edges.long(), torch.zeros((), dtype=torch.long, device=self.device))
        hit = (over[e] & valid).any(dim=1)
        unrouted = net_lens < 2
        return torch.nonzero(hit | unrouted).flatten()

    def _route_batched(self, acc, cost, idx, src_d, dst_d, boxes_d, full_box_d, order_rank, net_nodes,
                       net_edges, net_lens, delta):
        lib = _lib.load()
        cap = self.cfg.path_cap
        K = int(idx.numel())
        st = _stream()
        old_e = net_edges[idx].contiguous()
        old_l = net_lens[idx].contiguous()
        check(lib.orsp_commit_batch(K, ptr(old_e), ptr(old_l), cap, ptr(acc.usage), ptr(acc.present), -1, st),
              "orsp_commit_batch")
        s = src_d[idx].contiguous()
        t = dst_d[idx].contiguous()
        b = boxes_d[idx].contiguous()
        order = torch.argsort(order_rank[idx], stable=True).to(torch.int32)
        nodes, edges, lens = self.dg.batch_bbox(cost, s, t, b, order=order, delta=delta, path_cap=cap)
        if self.cfg.full_graph_retry:
            fail = torch.nonzero(lens < 2).flatten()
            if fail.numel() > 0:
                fb = full_box_d.expand(int(fail.numel()), 6).contiguous()
                n2, e2, l2 = self.dg.batch_bbox(cost, s[fail].contiguous(), t[fail].contiguous(), fb,
                                                delta=delta, path_cap=cap)
                nodes[fail] = n2
                edges[fail] = e2
                lens[fail] = l2
        bad = lens < 0
        if bool(bad.any()):
            raise _lib.OrspError(int(lens[bad][0]), "orsp_sssp_batch_bbox", "per-search failure status")
        net_nodes[idx] = nodes
        net_edges[idx] = edges
        net_lens[idx] = lens
        check(lib.orsp_commit_batch(K, ptr(edges), ptr(lens), cap, ptr(acc.usage), ptr(acc.present), 1, st),
              "orsp_commit_batch")

    def _route_sequential(self, acc, cost, idx, src, dst, boxes, net_nodes, net_edges, net_lens, delta):
        lib = _lib.load()
        cap = self.cfg.path_cap
        st = _stream()
        lens_h = net_lens.cpu().numpy()
        for k in idx.cpu().tolist():
            L = int(lens_h[k])
            if L >= 2:
                check(lib.orsp_commit_edges(L - 1, ptr(net_edges[k]), ptr(acc.usage), ptr(acc.present), -1, st),
                      "orsp_commit_edges")
            if self.cfg.roi == "bbox" and self.dg.is_lattice:
                g2r = "box"
                status, path, _ = self.dg.sssp_box(cost, int(src[k]), int(dst[k]), boxes[k], delta=delta,
                                                   path_cap=cap)
            else:
                if self.cfg.roi == "bbox":
                    g2r = self.roi.box_map(boxes[k])
                elif self.cfg.roi == "bfs":
                    _, g2r = self.roi.extract_roi(int(src[k]), int(dst[k]))
                else:
                    g2r = None
                status, path, _ = self.dg.sssp(cost, int(src[k]), int(dst[k]), roi_map=g2r, delta=delta,
                                               path_cap=cap)
            if (status != _lib.ORSP_OK or path is None or path.numel() < 2) and self.cfg.full_graph_retry \
                    and g2r is not None:
                status, path, _ = self.dg.sssp(cost, int(src[k]), int(dst[k]), roi_map=None, delta=delta,
                                               path_cap=cap)
            if status == _lib.ORSP_OK and path is not None and path.numel() >= 2:
                n = int(path.numel())
                e = self.dg.path_to_edges(path)
                net_nodes[k, :n] = path
                net_edges[k, : n - 1] = e
                net_lens[k] = n
                check(lib.orsp_commit_edges(n - 1, ptr(e), ptr(acc.usage), ptr(acc.present), 1, st),
                      "orsp_commit_edges")
            else:
                net_lens[k] = 0

    # ------------------------------------------------------------------ per-net costs
    def _live(self, acc, pres_fac, edges=None, n=0):
        cfg = self.cfg
        check(_lib.load().orsp_update_costs_live(self.E, ptr(edges), int(n), ptr(self.base), ptr(acc.usage),
                                                 ptr(acc.capacity), ptr(acc.history), float(pres_fac),
                                                 float(cfg.hist_cost_weight), float(cfg.via_cost_multiplier),
                                                 float(cfg.base_cost_weight), 1 if cfg.add_jitter else 0,
                                                 ptr(acc.total_cost), _stream()), "orsp_update_costs_live")

    def _live_paths(self, acc, pres_fac, edges, lens):
        cfg = self.cfg
        check(_lib.load().orsp_update_costs_live_paths(int(lens.numel()), ptr(edges), ptr(lens), int(edges.shape[1]),
                                                       ptr(self.base), ptr(acc.usage), ptr(acc.capacity),
                                                       ptr(acc.history), float(pres_fac), float(cfg.hist_cost_weight),
                                                       float(cfg.via_cost_multiplier), float(cfg.base_cost_weight),
                                                       1 if cfg.add_jitter else 0, ptr(acc.total_cost), _stream()),
              "orsp_update_costs_live_paths")

    def _route_nets_device(self, acc, pres_fac, order, groups, src, dst, boxes, net_nodes, net_edges, net_lens):
        """orsp_route_nets over `order` (host int32), cut into `groups` (host
        int32 group_ptr, or None for one net per group)."""
        cfg = self.cfg
        order = np.ascontiguousarray(order, dtype=np.int32)
        boxes_c = np.ascontiguousarray(boxes, dtype=np.int32)
        gp = None if groups is None else np.ascontiguousarray(groups, dtype=np.int32)
        check(_lib.load().orsp_route_nets(
            self.dg.handle, int(len(src)), ptr(src), ptr(dst), ptr(boxes_c), int(order.size), ptr(order),
            0 if gp is None else int(gp.size - 1), ptr(gp), ptr(net_nodes), ptr(net_edges), int(net_nodes.shape[1]),
            ptr(net_lens), ptr(acc.total_cost), ptr(self.base), ptr(acc.usage), ptr(acc.present), ptr(acc.capacity),
            ptr(acc.history), float(pres_fac), float(cfg.hist_cost_weight), float(cfg.via_cost_multiplier),
            float(cfg.base_cost_weight), 1 if cfg.add_jitter else 0, _stream()), "orsp_route_nets")

    def _route_nets_snapshot(self, acc, pres_fac, order, G, src, dst, boxes, net_nodes, net_edges, net_lens):
        """orsp_route_nets_snapshot over `order` (host int32) in groups of G
        consecutive nets, with cfg.group_repair repair rounds; returns the
        searches made."""
        cfg = self.cfg
        order = np.ascontiguousarray(order, dtype=np.int32)
        boxes_c = np.ascontiguousarray(boxes, dtype=np.int32)
        gp = np.ascontiguousarray(np.append(np.arange(0, order.size, G), order.size), dtype=np.int32)
        n = ctypes.c_int64(0)
        check(_lib.load().orsp_route_nets_snapshot(
            self.dg.handle, int(len(src)), ptr(src), ptr(dst), ptr(boxes_c), int(order.size), ptr(order),
            int(gp.size - 1), ptr(gp), int(max(0, cfg.group_repair)), ptr(net_nodes), ptr(net_edges),
            int(net_nodes.shape[1]), ptr(net_lens), ptr(acc.total_cost), ptr(self.base), ptr(acc.usage),
            ptr(acc.present), ptr(acc.capacity), ptr(acc.history), float(pres_fac), float(cfg.hist_cost_weight),
            float(cfg.via_cost_multiplier), float(cfg.base_cost_weight), 1 if cfg.add_jitter else 0,
            ctypes.byref(n), _stream()), "orsp_route_nets_snapshot")
        return int(n.value)

    def _route_net_sequential(self, acc, pres_fac, idx, src, dst, boxes, net_nodes, net_edges, net_lens, delta):
        if self.cfg.native_loop and self.dg.route_loop_ok:
            self._route_nets_device(acc, pres_fac, idx.cpu().numpy(), None, src, dst, boxes, net_nodes, net_edges,
                                    net_lens)
        else:
            self._route_net_sequential_host(acc, pres_fac, idx, src, dst, boxes, net_nodes, net_edges, net_lens,
                                            delta)

    def _route_net_sequential_host(self, acc, pres_fac, idx, src, dst, boxes, net_nodes, net_edges, net_lens,
                                   delta):
        """The same loop driven from the host, one net at a time (the plain
        form the device loop is checked against)."""
        lib = _lib.load()
        cap = self.cfg.path_cap
        st = _stream()
        cost = acc.total_cost
        lens_h = net_lens.cpu().numpy()
        for k in idx.cpu().tolist():
            L = int(lens_h[k])
            if L >= 2:
                old = net_edges[k, : L - 1]
                check(lib.orsp_commit_edges(L - 1, ptr(old), ptr(acc.usage), ptr(acc.present), -1, st),
                      "orsp_commit_edges")
                self._live(acc, pres_fac, old, L - 1)
            if self.dg.is_lattice:
                status, path, _ = self.dg.sssp_box(cost, int(src[k]), int(dst[k]), boxes[k], delta=delta,
                                                   path_cap=cap)
            else:
                g2r = self.roi.box_map(boxes[k])
                status, path, _ = self.dg.sssp(cost, int(src[k]), int(dst[k]), roi_map=g2r, delta=delta,
                                               path_cap=cap)
            if status == _lib.ORSP_OK and path is not None and path.numel() >= 2:
                n = int(path.numel())
                e = self.dg.path_to_edges(path)
                net_nodes[k, :n] = path
                net_edges[k, : n - 1] = e
                net_lens[k] = n
                lens_h[k] = n
                check(lib.orsp_commit_edges(n - 1, ptr(e), ptr(acc.usage), ptr(acc.present), 1, st),
                      "orsp_commit_edges")
                self._live(acc, pres_fac, e, n - 1)
            else:
                net_lens[k] = 0
                lens_h[k] = 0

    def _route_net_batched(self, acc, pres_fac, idx, src_d, dst_d, boxes_d, boxes, order_levels, net_nodes,
                           net_edges, net_lens, delta, src=None, dst=None):
        G = int(self.cfg.group_nets)
        if self.cfg.native_loop and self.dg.route_loop_ok and src is not None:
            idx_h = idx.cpu().numpy()
            if G > 0:
                n = self._route_nets_snapshot(acc, pres_fac, idx_h, G, src, dst, boxes, net_nodes, net_edges,
                                              net_lens)
                self._searches += n - int(idx_h.size)
                return
            order, groups = level_groups(idx_h, level_schedule(boxes[idx_h]))
            self._route_nets_device(acc, pres_fac, order, groups, src, dst, boxes, net_nodes, net_edges, net_lens)
            return
        lib = _lib.load()
        cap = self.cfg.path_cap
        st = _stream()
        cost = acc.total_cost
        idx_h = idx.cpu().numpy()
        if G > 0:  # snapshot groups: consecutive chunks of the order
            lv = (np.arange(len(idx_h)) // G).astype(np.int32)
        else:
            lv = level_schedule(boxes[idx_h])
        for L in range(int(lv.max()) + 1 if len(lv) else 0):
            sel = torch.from_numpy(idx_h[lv == L]).to(self.device)
            for rep in range(1 + (max(0, int(self.cfg.group_repair)) if G > 0 else 0)):
                if rep:
                    # repair: the nets whose path shares an edge with an
                    # earlier net of the same snapshot, searched again on the
                    # live costs (which now hold every path of the group)
                    sel = sel[self._group_conflicts(sel, net_edges, net_lens)]
                    if sel.numel() == 0:
                        break
                K = int(sel.numel())
                old_e = net_edges[sel].contiguous()
                old_l = net_lens[sel].contiguous()
                check(lib.orsp_commit_batch(K, ptr(old_e), ptr(old_l), cap, ptr(acc.usage), ptr(acc.present), -1,
                                            st), "orsp_commit_batch")
                self._live_paths(acc, pres_fac, old_e, old_l)
                nodes, edges, lens = self.dg.batch_bbox(cost, src_d[sel].contiguous(), dst_d[sel].contiguous(),
                                                        boxes_d[sel].contiguous(), delta=delta, path_cap=cap)
                if K and int(lens.min().item()) < 0:
                    bad = lens[lens < 0]
                    raise _lib.OrspError(int(bad[0]), "orsp_sssp_batch_bbox", "per-search failure status")
                net_nodes[sel] = nodes
                net_edges[sel] = edges
                net_lens[sel] = lens
                check(lib.orsp_commit_batch(K, ptr(edges), ptr(lens), cap, ptr(acc.usage), ptr(acc.present), 1, st),
                      "orsp_commit_batch")
                self._live_paths(acc, pres_fac, edges, lens)
                if rep:
                    self._searches += K

    def _group_conflicts(self, sel, net_edges, net_lens):
        """Mask over sel: the nets whose path uses an edge that an earlier net
        of sel (in sel's order) also uses."""
        n = int(sel.numel())
        cap = net_edges.shape[1]
        lens = net_lens[sel].long()
        valid = torch.arange(cap, device=self.device)[None, :] < (lens - 1).clamp_min(0)[:, None]
        e = net_edges[sel].long()[valid]
        r = torch.arange(n, device=self.device)[:, None].expand(n, cap)[valid]
        if self._owner is None or self._owner.numel() != self.E:
            self._owner = torch.full((self.E,), 1 << 30, dtype=torch.int64, device=self.device)
        own = self._owner
        own.scatter_reduce_(0, e, r, reduce="amin")
        hit = own[e] < r
        own[e] = 1 << 30
        conf = torch.zeros(n, dtype=torch.bool, device=self.device)
        conf[r[hit]] = True
        return conf

    # ------------------------------------------------------------------
    def route(self, src, dst, mode: str = "batched", history_init=None, callback=None) -> RouteResult:
        cfg = self.cfg
        if mode not in ("batched", "sequential"):
            raise ValueError("mode must be 'batched' or 'sequential'")
        if mode == "batched" and cfg.roi != "bbox":
            raise ValueError("the batched kernel searches box ROIs (roi='bbox')")
        dev = self.device
        torch.cuda.synchronize(dev)
        t_start = time.perf_counter()
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        M = len(src)
        cap = cfg.path_cap
        margins = np.full(M, cfg.roi_margin, dtype=np.int64)
        streak = np.zeros(M, dtype=np.int64)
        boxes = bbox_with_margin(self.lat, src, dst, margins)
        vol = (boxes[:, 1] - boxes[:, 0] + 1).astype(np.int64) * (boxes[:, 3] - boxes[:, 2] + 1) * \
            (boxes[:, 5] - boxes[:, 4] + 1)
        order_rank = torch.from_numpy(np.argsort(np.argsort(-vol, kind="stable"), kind="stable").astype(np.int64)).to(dev)
        src_d = torch.from_numpy(src).to(dev)
        dst_d = torch.from_numpy(dst).to(dev)
        boxes_d = torch.from_numpy(boxes).to(dev)
        full_box_d = torch.tensor([[0, self.lat.nx - 1, 0, self.lat.ny - 1, 0, self.lat.nz - 1]], dtype=torch.int32,
                                  device=dev)
        net_nodes = torch.zeros((M, cap), dtype=torch.int32, device=dev)
        net_edges = torch.full((M, cap), -1, dtype=torch.int32, device=dev)
        net_lens = torch.zeros(M, dtype=torch.int32, device=dev)
        acc = DeviceEdgeAccountant(self.E, device=dev)
        if history_init is not None:
            acc.history.copy_(as_device(history_init, torch.float32, dev))
        self.acc = acc
        all_idx = torch.arange(M, device=dev)
        pres_fac = cfg.pres_fac_init
        stats: List[IterationStats] = []
        converged = False
        if cfg.cost_update not in ("iteration", "net"):
            raise ValueError("cost_update must be 'iteration' or 'net'")
        net_policy = cfg.cost_update == "net"
        if net_policy and cfg.roi != "bbox":
            raise ValueError("per-net costs are implemented for box ROIs")
        acc.total_cost = torch.empty(self.E, dtype=torch.float32, device=dev)
        if cfg.batch_plan is not None:
            self.dg.set_batch_plan(cfg.batch_plan)
        if cfg.first_pass not in ("sequential", "independent"):
            raise ValueError("first_pass must be 'sequential' or 'independent'")
        for it in range(1, cfg.max_iterations + 1):
            t_it = time.perf_counter()
            searches0 = self._searches
            acc.refresh_from_canonical()
            if net_policy:
                self._live(acc, pres_fac)
            else:
                if it == 1:
                    acc.present_ema.copy_(acc.present)
                acc.update_present_ema(beta=cfg.present_ema_beta)
                acc.update_costs(self.base, pres_fac, cfg.hist_cost_weight, add_jitter=cfg.add_jitter,
                                 via_cost_multiplier=cfg.via_cost_multiplier, base_cost_weight=cfg.base_cost_weight)
            cost = acc.total_cost
            delta = cfg.delta if cfg.delta is not None else 0.0  # 0: chosen on the device
            off = None
            if it > 1 and (cfg.reroute != "all" or cfg.stall_grow > 0):
                off = self._offenders(acc, net_edges, net_lens, all_idx)
            idx = all_idx if (it == 1 or cfg.reroute == "all") else off
            if cfg.stall_grow > 0 and off is not None:
                # nets that offended stall_iterations times running get a wider box
                hit = np.zeros(M, dtype=bool)
                hit[off.cpu().numpy()] = True
                streak = np.where(hit, streak + 1, 0)
                grow = streak >= cfg.stall_iterations
                if grow.any():
                    margins[grow] += cfg.stall_grow
                    streak[grow] = 0
                    boxes = bbox_with_margin(self.lat, src, dst, margins)
                    boxes_d = torch.from_numpy(boxes).to(dev)
            if cfg.net_order == "disjoint" and idx.numel() > 1:
                idx = torch.from_numpy(disjoint_order(boxes, idx.cpu().numpy()).astype(np.int64)).to(dev)
            independent = net_policy and it == 1 and cfg.first_pass == "independent"
            if independent and idx.numel() > 0:
                # first pass: every net searched on the same (initial) costs,
                # then all committed - one batch launch in batched mode
                if mode == "batched":
                    self._route_batched(acc, cost, idx, src_d, dst_d, boxes_d, full_box_d, order_rank, net_nodes,
                                        net_edges, net_lens, delta)
                else:
                    self._route_sequential(acc, cost, idx, src, dst, boxes, net_nodes, net_edges, net_lens, delta)
            elif idx.numel() > 0 and net_policy:
                if mode == "batched":
                    self._route_net_batched(acc, pres_fac, idx, src_d, dst_d, boxes_d, boxes, order_rank, net_nodes,
                                            net_edges, net_lens, delta, src=src, dst=dst)
                else:
                    self._route_net_sequential(acc, pres_fac, idx, src, dst, boxes, net_nodes, net_edges, net_lens,
                                               delta)
            elif idx.numel() > 0:
                if mode == "batched":
                    self._route_batched(acc, cost, idx, src_d, dst_d, boxes_d, full_box_d, order_rank, net_nodes,
                                        net_edges, net_lens, delta)
                else:
                    self._route_sequential(acc, cost, idx, src, dst, boxes, net_nodes, net_edges, net_lens, delta)
            acc.refresh_from_canonical()
            over_sum, over_cnt = acc.compute_overuse()
            failed = int((net_lens < 2).sum().item())
            stats.append(IterationStats(it, pres_fac, M - failed, failed, over_sum, over_cnt,
                                        int(idx.numel()) + self._searches - searches0,
                                        time.perf_counter() - t_it))
            if callback is not None:
                callback(stats[-1])
            if over_sum == 0 and failed == 0:
                converged = True
                break
            gain = cfg.hist_gain
            if cfg.hist_gain_boost and it >= 8 and over_sum > 0:
                gain = min(1.2, cfg.hist_gain * 1.25)
            decay = cfg.history_decay if it >= cfg.history_decay_from else 1.0
            acc.update_history(gain, base_costs=self.base, history_cap_multiplier=cfg.history_cap_multiplier,
                               decay_factor=decay, use_raw_present=True)
            pres_fac = min(pres_fac * cfg.pres_fac_mult, cfg.pres_fac_max)
        torch.cuda.synchronize(dev)
        seconds = time.perf_counter() - t_start
        lens_h = net_lens.cpu().numpy()
        nodes_h = net_nodes.cpu().numpy()
        edges_h = net_edges.cpu().numpy()
        paths = [nodes_h[k, : lens_h[k]].copy() if lens_h[k] >= 2 else np.zeros(0, np.int32) for k in range(M)]
        all_e = np.concatenate([edges_h[k, : max(lens_h[k] - 1, 0)] for k in range(M)]) if M else np.zeros(0)
        all_e = all_e.astype(np.int64)
        vias = int(self.edge_kind[all_e].sum()) if all_e.size else 0
        wl = int(all_e.size - vias)
        return RouteResult(converged, stats, seconds, paths, acc.usage.cpu().numpy(), wl, vias,
                           meta={"mode": mode, "nets": M})
