"""ORACLE - test infrastructure only.

CPU restatement of the plain PathFinder loop that orthoroute_b200.negotiate
runs on the GPU (steps of PathFinderRouter._pathfinder_negotiation,
orthoroute/algorithms/manhattan/unified_pathfinder.py:3548-4259, and
_route_all, UPF:4441-4823): numpy float32 accounting in the reference's
expression order and the C heap Dijkstra on box ROIs.  Used to check that the
device loop gives bit-identical per-iteration overuse and final routes.  It
also restates the loop's snapshot-group schedule (cfg.group_nets /
group_repair: groups of nets searched on one cost snapshot, as the
reference's batched mode searches a batch of ROIs on one cost array,
CD:2014, then repair rounds for nets that share an edge with an earlier net
of the group), which orsp_route_nets_snapshot runs on the device.
"""
from __future__ import annotations

import time

import numpy as np

from . import orsp_oracle as O


def _first_fit_rounds(boxes, idx):
    """idx regrouped into rounds: a net joins the lowest round holding no box
    that meets its box; rounds concatenated in order."""
    rounds = []
    for k in idx:
        bk = boxes[k]
        for r in rounds:
            if not any(bk[0] <= boxes[q][1] and boxes[q][0] <= bk[1] and bk[2] <= boxes[q][3] and
                       boxes[q][2] <= bk[3] and bk[4] <= boxes[q][5] and boxes[q][4] <= bk[5] for q in r):
                r.append(k)
                break
        else:
            rounds.append([k])
    return np.array([k for r in rounds for k in r], dtype=np.int64)


def route_plain(lat, src, dst, cfg, base_cost=None, history_init=None, max_nets_per_iter=None):
    """Returns dict(trace=[(over_sum, over_cnt, failed)], paths=[...], usage, converged, seconds)."""
    from orthoroute_b200.lattice import bbox_with_margin  # pure numpy helper

    t0 = time.perf_counter()
    src = np.asarray(src, dtype=np.int32)
    dst = np.asarray(dst, dtype=np.int32)
    M = len(src)
    E = lat.E
    base = (lat.base_cost if base_cost is None else base_cost).astype(np.float32)
    cap_paths = cfg.path_cap
    margins = np.full(M, cfg.roi_margin, dtype=np.int64)
    streak = np.zeros(M, dtype=np.int64)
    boxes = bbox_with_margin(lat, src, dst, margins)
    stall_grow = getattr(cfg, "stall_grow", 0)
    net_order = getattr(cfg, "net_order", "index")
    full_box = np.array([[0, lat.nx - 1, 0, lat.ny - 1, 0, lat.nz - 1]], dtype=np.int32)
    usage = np.zeros(E, dtype=np.int64)
    capacity = np.ones(E, dtype=np.float32)
    present_ema = np.zeros(E, dtype=np.float32)
    history = np.zeros(E, dtype=np.float32) if history_init is None else history_init.astype(np.float32).copy()
    net_paths = [np.zeros(0, np.int32) for _ in range(M)]
    net_edges = [np.zeros(0, np.int32) for _ in range(M)]
    pres_fac = cfg.pres_fac_init
    trace = []
    converged = False
    net_policy = getattr(cfg, "cost_update", "iteration") == "net"
    jitter = (np.arange(E, dtype=np.float32) % 9973 * np.float32(1e-6)) if cfg.add_jitter else None
    adjusted = base * np.float32(cfg.via_cost_multiplier) * np.float32(cfg.base_cost_weight)

    def live_cost(e):
        """Live-usage cost of edges e (the GPU's orsp_update_costs_live)."""
        over = np.maximum(np.float32(0), (usage[e].astype(np.float32) + np.float32(1)) - capacity[e])
        t = (adjusted[e] + np.float32(pres_fac) * over) + np.float32(cfg.hist_cost_weight) * history[e]
        if jitter is not None:
            t = t + jitter[e]
        return t.astype(np.float32)

    def _snapshot_group(sel, repair):
        """Rip up every net of sel, recompute the costs of the freed edges,
        search all of sel on those costs, commit all and recompute the costs
        of the new edges; then up to `repair` rounds over the nets whose path
        uses an edge that an earlier net of the round also uses."""
        nonlocal cost
        sel = np.asarray(sel, dtype=np.int64)
        for rep in range(repair + 1):
            if rep:
                first = {}
                for j, k in enumerate(sel):
                    for e in net_edges[k].tolist():
                        first.setdefault(e, j)
                flag = np.array([any(first[e] < j for e in net_edges[k].tolist()) for j, k in enumerate(sel)],
                                dtype=bool)
                sel = sel[flag]
                if sel.size == 0:
                    return
            freed = [net_edges[k] for k in sel if net_edges[k].size]
            for e in freed:
                np.subtract.at(usage, e, 1)
                np.maximum(usage, 0, out=usage)
            if freed:
                fe = np.concatenate(freed)
                cost[fe] = live_cost(fe)
            nodes, lens = O.batch_bbox(lat.indptr, lat.indices, cost, lat.nx, lat.ny, lat.nz, src[sel], dst[sel],
                                       boxes[sel], cap_paths)
            new = []
            for j, k in enumerate(sel):
                L = int(lens[j])
                if L >= 2:
                    p = nodes[j, :L].copy()
                    net_paths[k] = p
                    net_edges[k] = O.path_to_edges(lat.indptr, lat.indices, p)
                    np.add.at(usage, net_edges[k], 1)
                    new.append(net_edges[k])
                else:
                    net_paths[k] = np.zeros(0, np.int32)
                    net_edges[k] = np.zeros(0, np.int32)
            if new:
                ne = np.concatenate(new)
                cost[ne] = live_cost(ne)

    cost = None
    for it in range(1, cfg.max_iterations + 1):
        if net_policy:
            cost = live_cost(np.arange(E))
            over_e = usage.astype(np.float32) > capacity
            off = np.array([k for k in range(M) if len(net_paths[k]) < 2 or over_e[net_edges[k]].any()],
                           dtype=np.int64)
            idx = np.arange(M) if (it == 1 or cfg.reroute == "all") else off
            if stall_grow > 0 and it > 1:
                # a net offending stall_iterations times running: margin += stall_grow
                offset = set(off.tolist())
                for k in range(M):
                    streak[k] = streak[k] + 1 if k in offset else 0
                    if streak[k] >= cfg.stall_iterations:
                        margins[k] += stall_grow
                        streak[k] = 0
                boxes = bbox_with_margin(lat, src, dst, margins)
            if net_order == "disjoint":
                idx = _first_fit_rounds(boxes, idx)
            if it == 1 and getattr(cfg, "first_pass", "sequential") == "independent":
                # first pass: every net on the initial costs, then all committed
                nodes, lens = O.batch_bbox(lat.indptr, lat.indices, cost, lat.nx, lat.ny, lat.nz, src[idx], dst[idx],
                                           boxes[idx], cap_paths)
                for j, k in enumerate(idx):
                    L = int(lens[j])
                    if L >= 2:
                        p = nodes[j, :L].copy()
                        net_paths[k] = p
                        net_edges[k] = O.path_to_edges(lat.indptr, lat.indices, p)
                        np.add.at(usage, net_edges[k], 1)
                    else:
                        net_paths[k] = np.zeros(0, np.int32)
                        net_edges[k] = np.zeros(0, np.int32)
                idx = np.zeros(0, np.int64)
            G = int(getattr(cfg, "group_nets", 0))
            if G > 0:
                # snapshot groups of G consecutive nets, then repair rounds
                for a in range(0, len(idx), G):
                    _snapshot_group(idx[a:a + G], max(0, int(getattr(cfg, "group_repair", 0))))
                idx = np.zeros(0, np.int64)
            for k in idx:  # sequential: rip up, search on live costs, commit
                e = net_edges[k]
                if e.size:
                    np.subtract.at(usage, e, 1)
                    np.maximum(usage, 0, out=usage)
                    cost[e] = live_cost(e)
                nodes, lens = O.batch_bbox(lat.indptr, lat.indices, cost, lat.nx, lat.ny, lat.nz, src[k:k + 1],
                                           dst[k:k + 1], boxes[k:k + 1], cap_paths)
                L = int(lens[0])
                if L >= 2:
                    p = nodes[0, :L].copy()
                    en = O.path_to_edges(lat.indptr, lat.indices, p)
                    net_paths[k] = p
                    net_edges[k] = en
                    np.add.at(usage, en, 1)
                    cost[en] = live_cost(en)
                else:
                    net_paths[k] = np.zeros(0, np.int32)
                    net_edges[k] = np.zeros(0, np.int32)
            present = usage.astype(np.float32)
            over_sum, over_cnt = O.compute_overuse(present, capacity)
            failed = sum(1 for p in net_paths if len(p) < 2)
            trace.append((over_sum, over_cnt, failed))
            if over_sum == 0 and failed == 0:
                converged = True
                break
            gain = cfg.hist_gain
            if cfg.hist_gain_boost and it >= 8 and over_sum > 0:
                gain = min(1.2, cfg.hist_gain * 1.25)
            decay = cfg.history_decay if it >= cfg.history_decay_from else 1.0
            history = O.update_history(history, present, capacity, gain, base_costs=base,
                                       history_cap_multiplier=cfg.history_cap_multiplier, decay_factor=decay)
            pres_fac = min(pres_fac * cfg.pres_fac_mult, cfg.pres_fac_max)
            continue
        present = usage.astype(np.float32)
        if it == 1:
            present_ema = present.copy()
        present_ema = O.update_present_ema(present, present_ema, beta=cfg.present_ema_beta)
        cost = O.update_costs(base, present_ema, capacity, history, pres_fac, cfg.hist_cost_weight,
                              add_jitter=cfg.add_jitter, via_cost_multiplier=cfg.via_cost_multiplier,
                              base_cost_weight=cfg.base_cost_weight)
        if it == 1 or cfg.reroute == "all":
            idx = np.arange(M)
        else:
            over_e = present > capacity
            idx = np.array([k for k in range(M) if len(net_paths[k]) < 2 or over_e[net_edges[k]].any()],
                           dtype=np.int64)
        if idx.size:
            for k in idx:  # rip up
                e = net_edges[k]
                if e.size:
                    np.subtract.at(usage, e, 1)
                    np.maximum(usage, 0, out=usage)
            nodes, lens = O.batch_bbox(lat.indptr, lat.indices, cost, lat.nx, lat.ny, lat.nz, src[idx], dst[idx],
                                       boxes[idx], cap_paths)
            if cfg.full_graph_retry:
                fail = np.nonzero(lens < 2)[0]
                if fail.size:
                    n2, l2 = O.batch_bbox(lat.indptr, lat.indices, cost, lat.nx, lat.ny, lat.nz, src[idx][fail],
                                          dst[idx][fail], np.repeat(full_box, fail.size, axis=0), cap_paths)
                    nodes[fail] = n2
                    lens[fail] = l2
            for j, k in enumerate(idx):
                L = int(lens[j])
                if L >= 2:
                    p = nodes[j, :L].copy()
                    e = O.path_to_edges(lat.indptr, lat.indices, p)
                    net_paths[k] = p
                    net_edges[k] = e
                    np.add.at(usage, e, 1)
                else:
                    net_paths[k] = np.zeros(0, np.int32)
                    net_edges[k] = np.zeros(0, np.int32)
        present = usage.astype(np.float32)
        over_sum, over_cnt = O.compute_overuse(present, capacity)
        failed = sum(1 for p in net_paths if len(p) < 2)
        trace.append((over_sum, over_cnt, failed))
        if over_sum == 0 and failed == 0:
            converged = True
            break
        gain = cfg.hist_gain
        if cfg.hist_gain_boost and it >= 8 and over_sum > 0:
            gain = min(1.2, cfg.hist_gain * 1.25)
        decay = cfg.history_decay if it >= cfg.history_decay_from else 1.0
        history = O.update_history(history, present, capacity, gain, base_costs=base,
                                   history_cap_multiplier=cfg.history_cap_multiplier, decay_factor=decay)
        pres_fac = min(pres_fac * cfg.pres_fac_mult, cfg.pres_fac_max)
    return {
        "trace": trace,
        "paths": net_paths,
        "usage": usage.astype(np.int32),
        "converged": converged,
        "seconds": time.perf_counter() - t0,
        "history": history,
    }
