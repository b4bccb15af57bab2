"""Per-iteration negotiation bookkeeping with the data-parallel parts on the
GPU (orsp_bookkeeping.cu) and the selection logic of the reference on the
host, so that the results are the reference's:

* ``rebuild_node_owner``      PathFinderRouter._rebuild_node_owner (UPF:2762-2837)
* ``detect_barrel_conflicts`` PathFinderRouter._detect_barrel_conflicts (UPF:5478-5569)
* ``apply_barrel_penalty``    the Phase-1 penalty of _pathfinder_negotiation (UPF:3852-3871)
* ``order_nets_by_difficulty`` PathFinderRouter._order_nets_by_difficulty (UPF:4401-4439)
* ``build_hotset``            PathFinderRouter._build_hotset (UPF:5009-5140)

UPF = orthoroute/algorithms/manhattan/unified_pathfinder.py.  Nets are named
(the reference's net ids) and listed in the router's dict order; the random
draws use Python's random module exactly as the reference does (the global
generator for the difficulty rotation, random.Random(42 + iteration) for the
hotset sample), so a caller that seeds them the same way gets the same nets.
"""
from __future__ import annotations

import ctypes
import random
from typing import Dict, List, Optional, Sequence, Set, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .solver import DeviceGraph, _stream


def _pack(lists: Sequence[Sequence[int]], device) -> Tuple[torch.Tensor, torch.Tensor]:
    off = np.zeros(len(lists) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in lists])
    flat = np.fromiter((v for x in lists for v in x), dtype=np.int32, count=int(off[-1]))
    return (torch.from_numpy(flat if flat.size else np.zeros(1, np.int32)).to(device),
            torch.from_numpy(off).to(device))


class Bookkeeper:
    """The bookkeeping state of one routing run: net ids assigned on first
    use (_get_net_id, UPF:2839-2844) and the node-owner array."""

    def __init__(self, dg: DeviceGraph):
        self.dg = dg
        self.net_id_map: Dict[str, int] = {}
        self.next_net_id = 0
        self.node_owner = torch.full((dg.N,), -1, dtype=torch.int32, device=dg.device)

    def net_id(self, name: str) -> int:
        if name not in self.net_id_map:
            self.net_id_map[name] = self.next_net_id
            self.next_net_id += 1
        return self.net_id_map[name]

    # ------------------------------------------------------------- barrels
    def rebuild_node_owner(self, net_paths: Dict[str, Sequence[int]],
                           keepouts: Sequence[Tuple[int, int, int, str]] = ()) -> torch.Tensor:
        """Ownership from the committed paths' via barrels (dict order, last
        net wins) and then the escape-via keepouts [(z, x, y, net)] in dict
        order (z > 0, free nodes only, first entry wins).  Net ids are
        assigned on first use in that order."""
        items = [(n, p) for n, p in net_paths.items() if p is not None and len(p) >= 2]
        ids = np.array([self.net_id(n) for n, _ in items], np.int32)
        keep = [(z, x, y, n) for z, x, y, n in keepouts if z > 0]
        k_nodes = np.array([(z * self.dg.ny + y) * self.dg.nx + x for z, x, y, _ in keep], np.int32)
        k_ids = np.array([self.net_id(n) for _, _, _, n in keep], np.int32)
        paths, off = _pack([p for _, p in items], self.dg.device)
        dev = self.dg.device
        ids_d = torch.from_numpy(ids if ids.size else np.zeros(1, np.int32)).to(dev)
        kn_d = torch.from_numpy(k_nodes if k_nodes.size else np.zeros(1, np.int32)).to(dev)
        ki_d = torch.from_numpy(k_ids if k_ids.size else np.zeros(1, np.int32)).to(dev)
        check(_lib.load().orsp_node_owner(self.dg.handle, len(items), ptr(paths), ptr(off), ptr(ids_d), len(keep),
                                          ptr(kn_d), ptr(ki_d), ptr(self.node_owner), _stream()), "orsp_node_owner")
        return self.node_owner

    def detect_barrel_conflicts(self, net_edges: Dict[str, Sequence[int]]) -> Tuple[torch.Tensor, int]:
        """(uint8[E] mask of conflicting edges, conflict count with
        duplicates).  net_edges: the committed edge lists (path -> edges) of
        the nets, dict order."""
        items = [(n, e) for n, e in net_edges.items() if e is not None and len(e) > 0]
        ids = np.array([self.net_id(n) for n, _ in items], np.int32)
        edges, off = _pack([e for _, e in items], self.dg.device)
        ids_d = torch.from_numpy(ids if ids.size else np.zeros(1, np.int32)).to(self.dg.device)
        mask = torch.empty(self.dg.E, dtype=torch.uint8, device=self.dg.device)
        cnt = ctypes.c_int64(0)
        check(_lib.load().orsp_barrel_conflicts(self.dg.handle, len(items), ptr(edges), ptr(off), ptr(ids_d),
                                                ptr(self.node_owner), ptr(mask), ctypes.byref(cnt), _stream()),
              "orsp_barrel_conflicts")
        return mask, int(cnt.value)


def apply_barrel_penalty(present: torch.Tensor, mask: torch.Tensor, pres_fac: float) -> float:
    """present[conflicts] += min(10 pres_fac, 100) (once per edge); returns
    the penalty."""
    penalty = min(10.0 * pres_fac, 100.0)
    check(_lib.load().orsp_barrel_penalty(present.numel(), ptr(mask), ptr(present), float(penalty), _stream()),
          "orsp_barrel_penalty")
    return penalty


def net_scores(dg: DeviceGraph, net_edges: Sequence[Sequence[int]], present, capacity, history):
    """(congestion float64[M], impact float64[M], offender bool[M], hot edge count)."""
    M = len(net_edges)
    edges, off = _pack(net_edges, dg.device)
    cong = torch.empty(max(M, 1), dtype=torch.float64, device=dg.device)
    imp = torch.empty(max(M, 1), dtype=torch.float64, device=dg.device)
    offn = torch.empty(max(M, 1), dtype=torch.uint8, device=dg.device)
    hot = ctypes.c_int64(0)
    check(_lib.load().orsp_net_scores(dg.handle, M, ptr(edges), ptr(off), ptr(present), ptr(capacity),
                                      ptr(history), ptr(cong), ptr(imp), ptr(offn), ctypes.byref(hot), _stream()),
          "orsp_net_scores")
    return cong[:M].cpu().numpy(), imp[:M].cpu().numpy(), offn[:M].cpu().numpy().astype(bool), int(hot.value)


def difficulty_order(tasks: Dict[str, Tuple[int, int]], congestion: Dict[str, float], nx: int, ny: int) -> List[str]:
    """Host part of _order_nets_by_difficulty: hardest first by
    manhattan(src, dst) * 3 * (congestion + 1), ties by net id, then a
    rotation by random.randint(0, min(5, len // 10)) from the global random
    module.  congestion: the nets that have edges."""
    plane = nx * ny
    scores = []
    for n, (s, d) in tasks.items():
        sz, sr = divmod(int(s), plane)
        dz, dr = divmod(int(d), plane)
        sy, sx = divmod(sr, nx)
        dy, dx = divmod(dr, nx)
        distance = abs(dx - sx) + abs(dy - sy) + abs(dz - sz)
        scores.append((distance * (2 + 1) * (congestion.get(n, 0.0) + 1), n))
    scores.sort(reverse=True)
    rotation = random.randint(0, min(5, len(scores) // 10))
    ordered = [n for _, n in scores]
    if rotation > 0:
        ordered = ordered[rotation:] + ordered[:rotation]
    return ordered


def select_hotset(tasks: Dict[str, Tuple[int, int]], names: List[str], impact, offender, hot_count: int,
                  routed: Set[str], iteration: int, clean_iters: Dict[str, int], last_reroute: Dict[str, int],
                  hotset_cap: int = 512, freeze_after_clean: int = 3, ripped: Optional[Set[str]] = None) -> Set[str]:
    """Host part of _build_hotset, from the per-net scores of the nets that
    have edges (names, impact, offender) and the number of hot edges."""
    ripped = set() if ripped is None else set(ripped)
    if hot_count == 0:
        unrouted = {n for n in tasks if n not in routed}
        return unrouted | ripped
    offenders = {n for n, o in zip(names, offender) if o}
    for n in tasks:
        if n in offenders:
            clean_iters[n] = 0
        else:
            clean_iters[n] = clean_iters.get(n, 0) + 1
    frozen = {n for n in offenders if clean_iters.get(n, 0) >= freeze_after_clean}
    offenders -= frozen
    offenders |= ripped
    unrouted = {n for n in tasks if n not in routed}
    imp = dict(zip(names, (float(v) for v in impact)))
    scores = [(imp[n], n) for n in offenders if n in imp]
    for n in unrouted:
        if n not in offenders:
            scores.append((0.0, n))
    scores.sort(reverse=True)
    cap = min(hotset_cap, 100)
    rng = random.Random(42 + iteration)
    k_top = int(0.6 * cap)
    top = [n for _, n in scores[:k_top]]
    rest = [n for _, n in scores[k_top:]]
    k_rand = min(cap - k_top, len(rest))
    sample = rng.sample(rest, k_rand) if rest else []
    kept = [n for n in top + sample if iteration - last_reroute.get(n, -999) > 1]
    for n in kept:
        last_reroute[n] = iteration
    return set(kept)


def order_nets_by_difficulty(dg: DeviceGraph, tasks: Dict[str, Tuple[int, int]], net_to_edges: Dict[str, List[int]],
                             present, capacity, history, nx: int, ny: int) -> List[str]:
    """_order_nets_by_difficulty with the per-net congestion on the GPU."""
    names = list(net_to_edges.keys())
    cong, _, _, _ = net_scores(dg, [net_to_edges[n] for n in names], present, capacity, history)
    return difficulty_order(tasks, dict(zip(names, (float(v) for v in cong))), nx, ny)


def build_hotset(dg: DeviceGraph, tasks: Dict[str, Tuple[int, int]], net_to_edges: Dict[str, List[int]],
                 routed: Set[str], present, capacity, history, iteration: int, clean_iters: Dict[str, int],
                 last_reroute: Dict[str, int], hotset_cap: int = 512, freeze_after_clean: int = 3,
                 ripped: Optional[Set[str]] = None) -> Set[str]:
    """_build_hotset with the per-net scores on the GPU.  clean_iters and
    last_reroute are updated in place, as the reference's attributes."""
    names = list(net_to_edges.keys())
    _, impact, offender, hot_count = net_scores(dg, [net_to_edges[n] for n in names], present, capacity, history)
    return select_hotset(tasks, names, impact, offender, hot_count, routed, iteration, clean_iters, last_reroute,
                         hotset_cap, freeze_after_clean, ripped)
