"""ORACLE - test infrastructure only: the recorder of reference-router tapes
and the CPU oracle behind the replay interface of orthoroute_b200.tape.

Recording (needs the reference source tree; see tests/golden/
make_golden_dropin.py): ``TapeRecorder`` wraps the hooks of an initialised
PathFinderRouter and records, in order, every call into the hot path with its
inputs, outputs and the reference's time, plus the writes the negotiation
loop made to the accountant's arrays and canonical dict outside those
methods (``present.fill(0)``, ``pres[idx] += penalty``, ``present_ema =
present.copy()``, UPF:3651, 3868-3871, 4971-4985) as sparse diffs.  Each
search is also answered by the fp32 C oracle at record time; where the
reference's float64 sums pick another path, the oracle's is stored beside it.

``OracleBackend`` answers a replay with the oracle restatements (CPU), which
pins the oracle on the reference's real call stream.
"""
from __future__ import annotations

import inspect
import time

import numpy as np

from orthoroute_b200.tape import ACCT_ARRAYS, Tape, digest  # noqa: F401

# ----------------------------------------------------------------------------
# recording

class _Proxy:
    """Forwards attribute reads and writes to `target`, except the names in
    `override`."""

    def __init__(self, target, override):
        object.__setattr__(self, "_t", target)
        object.__setattr__(self, "_o", override)

    def __getattr__(self, name):
        o = object.__getattribute__(self, "_o")
        if name in o:
            return o[name]
        return getattr(object.__getattribute__(self, "_t"), name)

    def __setattr__(self, name, value):
        setattr(object.__getattribute__(self, "_t"), name, value)


class TapeRecorder:
    """Wraps the hooks of an initialised reference router (see module doc)."""

    def __init__(self, router, indptr, indices, oracle=None):
        self.tape = Tape()
        self.router = router
        self.acct = router.accounting
        self.indptr = np.asarray(indptr)
        self.indices = np.asarray(indices)
        self.oracle = oracle
        self.N = len(self.indptr) - 1
        self._snap = {n: self._arr(n) for n in ACCT_ARRAYS}
        self._canon = dict(self.acct.canonical)
        self._last_roi = None
        self._last_path = None
        self.it = 0
        self._install()

    # --- state tracking ---------------------------------------------------
    def _arr(self, name):
        v = getattr(self.acct, name, None)
        return None if v is None else np.array(v, dtype=np.float32, copy=True)

    def _sync_external(self):
        """Records the loop's own writes to the accountant since the last call."""
        for name in ACCT_ARRAYS:
            cur = getattr(self.acct, name, None)
            old = self._snap[name]
            if cur is None and old is None:
                continue
            cur = np.asarray(cur, dtype=np.float32)
            if old is None or old.shape != cur.shape:
                self.tape.events.append({"k": "full", "name": name, "val": self.tape.blob(cur)})
            else:
                diff = np.nonzero(old.view(np.uint32) != cur.view(np.uint32))[0]
                if diff.size == 0:
                    continue
                if diff.size > cur.size // 4:
                    self.tape.events.append({"k": "full", "name": name, "val": self.tape.blob(cur)})
                else:
                    self.tape.events.append({"k": "set", "name": name, "idx": self.tape.blob(diff, np.int64),
                                             "val": self.tape.blob(cur[diff])})
            self._snap[name] = cur.copy()
        if self.acct.canonical != self._canon:
            items = sorted(self.acct.canonical.items())
            k = np.array([i for i, _ in items], dtype=np.int64)
            v = np.array([c for _, c in items], dtype=np.int64)
            self.tape.events.append({"k": "canon", "keys": self.tape.blob(k), "vals": self.tape.blob(v)})
            self._canon = dict(self.acct.canonical)

    def _after(self, ev):
        ev["after"] = {}
        for name in ACCT_ARRAYS:
            a = self._arr(name)
            self._snap[name] = a
            ev["after"][name] = digest(a)
        self._canon = dict(self.acct.canonical)

    def _enc(self, v):
        if v is None or isinstance(v, (bool, int, float, str)):
            return v
        if isinstance(v, (np.integer,)):
            return int(v)
        if isinstance(v, (np.floating,)):
            return float(v)
        if isinstance(v, (list, tuple)) and all(isinstance(x, (int, np.integer)) for x in v):
            return {"blob": self.tape.blob(np.asarray(v, dtype=np.int64))}
        if isinstance(v, (list, tuple)):
            return [self._enc(x) for x in v]
        a = np.asarray(v)
        return {"blob": self.tape.blob(a)}

    def _router_state(self, names):
        out = {}
        for n in names:
            if hasattr(self.router, n) and getattr(self.router, n) is not None:
                out[n] = self.tape.blob(np.asarray(getattr(self.router, n)))
        return out

    # --- wrappers -----------------------------------------------------------
    def _install(self):
        acct = self.acct
        over = {}
        for m in ("refresh_from_canonical", "commit_path", "clear_path", "compute_overuse", "update_present_ema",
                  "update_history", "update_costs", "verify_present_matches_canonical"):
            over[m] = self._wrap_acct(m, getattr(acct, m))
        self.router.accounting = _Proxy(acct, over)
        ex = self.router.roi_extractor
        self.router.roi_extractor = _Proxy(ex, {"extract_roi": self._wrap_roi(ex.extract_roi)})
        s = self.router.solver
        s.find_path_roi = self._wrap_search(s.find_path_roi)
        s.find_path_multisource_multisink = self._refuse("find_path_multisource_multisink")
        self.router._path_to_edges = self._wrap_p2e(self.router._path_to_edges)
        self.router._apply_via_pooling_penalties = self._wrap_via_pen(self.router._apply_via_pooling_penalties)
        self.router._block_via_edges_with_collisions = self._wrap_via_block(
            self.router._block_via_edges_with_collisions)

    def _refuse(self, name):
        def f(*a, **k):
            raise RuntimeError(f"{name} is not recorded (portal runs are not taped)")
        return f

    def _wrap_acct(self, name, fn):
        sig = inspect.signature(fn)

        def w(*args, **kw):
            self._sync_external()
            b = sig.bind(*args, **kw)
            b.apply_defaults()
            ev = {"k": "acct", "m": name, "it": self.it}
            a = {}
            for key, v in b.arguments.items():
                if key == "router_instance":
                    a[key] = self._router_state(("via_col_use", "via_col_cap", "via_seg_use", "via_seg_cap")) \
                        if v is not None else None
                elif key == "edge_indices":
                    a[key] = {"blob": self.tape.blob(np.asarray(list(v), dtype=np.int64))}
                else:
                    a[key] = self._enc(v)
            ev["args"] = a
            t0 = time.perf_counter()
            out = fn(*args, **kw)
            ev["sec"] = time.perf_counter() - t0
            ev["out"] = self._enc(out) if not isinstance(out, tuple) else [self._enc(x) for x in out]
            self._after(ev)
            self.tape.events.append(ev)
            return out
        return w

    def _wrap_roi(self, fn):
        def w(src, dst, initial_radius=40, stagnation_bonus=0.0, portal_seeds=None):
            self._sync_external()
            t0 = time.perf_counter()
            roi, g2r = fn(src, dst, initial_radius=initial_radius, stagnation_bonus=stagnation_bonus,
                          portal_seeds=portal_seeds)
            sec = time.perf_counter() - t0
            self._last_roi = roi
            self.tape.events.append({"k": "roi", "it": self.it, "src": int(src), "dst": int(dst),
                                     "initial_radius": int(initial_radius),
                                     "stagnation_bonus": float(stagnation_bonus),
                                     "portal_seeds": None if not portal_seeds else
                                     [[int(n), float(c)] for n, c in portal_seeds],
                                     "len": int(len(roi)), "roi": digest(np.asarray(roi, dtype=np.int32)),
                                     "sec": sec})
            return roi, g2r
        return w

    def _wrap_search(self, fn):
        def w(src, dst, costs, roi_nodes, global_to_roi):
            self._sync_external()
            ev = {"k": "search", "it": self.it, "src": int(src), "dst": int(dst)}
            total = getattr(self.acct, "total_cost", None)
            ev["costs"] = "total" if costs is total else {"blob": self.tape.blob(np.asarray(costs, np.float32))}
            ev["costs_digest"] = digest(np.asarray(costs, np.float32))
            roi = np.asarray(roi_nodes, dtype=np.int32)
            if roi_nodes is self._last_roi:
                ev["roi"] = "last"
            elif roi.size == self.N and np.array_equal(roi, np.arange(self.N, dtype=np.int32)):
                ev["roi"] = "full"
            else:
                ev["roi"] = {"blob": self.tape.blob(roi)}
            ev["roi_digest"] = digest(roi)
            t0 = time.perf_counter()
            p = fn(src, dst, costs, roi_nodes, global_to_roi)
            ev["sec"] = time.perf_counter() - t0
            path = [int(x) for x in p] if p else None
            ev["out"] = path
            if self.oracle is not None:
                g2r = np.full(self.N, -1, np.int32)
                g2r[roi] = np.arange(roi.size, dtype=np.int32)
                q, *_ = self.oracle.dijkstra(self.indptr, self.indices, np.asarray(costs, np.float32), [int(src)],
                                             dst=int(dst), roi_map=g2r)
                q = q.tolist() if len(q) > 1 else None
                if q != path:
                    ev["oracle"] = q
            self._last_path = p
            self.tape.events.append(ev)
            return p
        return w

    def _wrap_p2e(self, fn):
        def w(path):
            self._sync_external()
            ev = {"k": "p2e", "it": self.it}
            ev["path"] = "last" if path is self._last_path else [int(x) for x in path]
            t0 = time.perf_counter()
            out = fn(path)
            ev["sec"] = time.perf_counter() - t0
            ev["out"] = [int(e) for e in out]
            self.tape.events.append(ev)
            return out
        return w

    def _wrap_via_pen(self, fn):
        def w(pres_fac):
            self._sync_external()
            r = self.router
            ev = {"k": "via_pen", "it": self.it, "pres_fac": float(pres_fac),
                  "state": self._router_state(("via_col_pres", "via_seg_pres", "via_seg_prefix", "layer_bias")),
                  "has_meta": getattr(r, "_via_edge_metadata", None) is not None,
                  "col_w": float(getattr(r.config, "via_column_weight", 1.0)),
                  "seg_w": float(getattr(r.config, "via_segment_weight", 1.0)),
                  "hot": float(getattr(r.config, "via_hot_layer_discount", 0.20))}
            t0 = time.perf_counter()
            out = fn(pres_fac)
            ev["sec"] = time.perf_counter() - t0
            self._after(ev)
            self.tape.events.append(ev)
            return out
        return w

    def _wrap_via_block(self, fn):
        def w():
            self._sync_external()
            r = self.router
            ev = {"k": "via_block", "it": self.it,
                  "state": self._router_state(("via_col_use", "via_col_cap", "via_seg_use", "via_seg_cap")),
                  "has_meta": getattr(r, "_via_edge_metadata", None) is not None}
            t0 = time.perf_counter()
            out = fn()
            ev["sec"] = time.perf_counter() - t0
            self._after(ev)
            self.tape.events.append(ev)
            return out
        return w

    def iteration_done(self, it, over_sum, over_cnt):
        self._sync_external()
        self.tape.events.append({"k": "iter", "it": int(it), "over_sum": int(over_sum), "over_cnt": int(over_cnt)})
        self.it = int(it)


# ----------------------------------------------------------------------------
# the oracle backend (CPU)

class OracleAccountant:
    """EdgeAccountant restated with the oracle's numpy functions (CPU)."""

    def __init__(self, E):
        self.E = int(E)
        self.canonical = {}
        self.use_gpu = False
        self.present = np.zeros(E, np.float32)
        self.present_ema = np.zeros(E, np.float32)
        self.history = np.zeros(E, np.float32)
        self.capacity = np.ones(E, np.float32)
        self.total_cost = None

    def refresh_from_canonical(self):
        self.present.fill(0)
        for i, c in self.canonical.items():
            if 0 <= i < self.E:
                self.present[i] = float(c)

    def commit_path(self, edge_indices):
        for i in edge_indices:
            self.canonical[i] = self.canonical.get(i, 0) + 1
            self.present[i] = self.present[i] + 1

    def clear_path(self, edge_indices):
        for i in edge_indices:
            if i in self.canonical:
                self.canonical[i] -= 1
                if self.canonical[i] <= 0:
                    del self.canonical[i]
            self.present[i] = np.maximum(0, self.present[i] - 1)

    def verify_present_matches_canonical(self):
        rec = np.zeros(self.E, np.float32)
        for i, c in self.canonical.items():
            if 0 <= i < self.E:
                rec[i] = float(c)
        return bool(np.sum(np.abs(self.present - rec)) <= 0.01)

    def compute_overuse(self, router_instance=None):
        from . import orsp_oracle as O

        s, c = O.compute_overuse(self.present, self.capacity)
        if router_instance is not None:
            for use, cap in (("via_col_use", "via_col_cap"), ("via_seg_use", "via_seg_cap")):
                if hasattr(router_instance, use) and hasattr(router_instance, cap):
                    s += int(np.maximum(0, getattr(router_instance, use) - getattr(router_instance, cap)).sum())
        return s, c

    def update_present_ema(self, beta=0.60):
        from . import orsp_oracle as O

        self.present_ema = O.update_present_ema(self.present, self.present_ema, beta)

    def update_history(self, gain, base_costs=None, history_cap_multiplier=10.0, decay_factor=0.98,
                       use_raw_present=False):
        from . import orsp_oracle as O

        pres = self.present if use_raw_present else self.present_ema
        self.history = O.update_history(self.history, pres, self.capacity, gain, base_costs,
                                        history_cap_multiplier, decay_factor)

    def update_costs(self, base_costs, pres_fac, hist_weight=1.0, add_jitter=True, via_cost_multiplier=1.0,
                     base_cost_weight=0.01, edge_layer=None, layer_bias_per_layer=None, edge_kind=None):
        from . import orsp_oracle as O

        self.total_cost = O.update_costs(base_costs, self.present_ema, self.capacity, self.history, pres_fac,
                                         hist_weight, add_jitter, via_cost_multiplier, base_cost_weight,
                                         edge_layer, layer_bias_per_layer, edge_kind)


class OracleBackend:
    """The CPU oracle behind the replay interface."""

    def __init__(self, indptr, indices, nx, ny, nz, max_roi_nodes=50_000):
        from . import orsp_oracle as O

        self.O = O
        self.indptr = np.asarray(indptr, np.int32)
        self.indices = np.asarray(indices, np.int32)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.acct = OracleAccountant(len(self.indices))
        self.meta = O.via_edge_metadata(self.indptr, self.indices, nx, ny, nz)
        self.max_roi_nodes = max_roi_nodes

    def extract_roi(self, src, dst, initial_radius, stagnation_bonus, portal_seeds):
        plane = self.nx * self.ny
        sx, sy = (src % plane) % self.nx, (src % plane) // self.nx
        dx, dy = (dst % plane) % self.nx, (dst % plane) // self.nx
        radius = max(60, int((abs(dx - sx) + abs(dy - sy)) * 0.75 + stagnation_bonus * 2.0))
        depth = min(int(radius + stagnation_bonus * 2.0), 150)
        keep = [n for n, _ in portal_seeds] if portal_seeds else None
        return self.O.roi_bfs(self.indptr, self.indices, src, dst, depth, self.max_roi_nodes, keep=keep)

    def find_path_roi(self, src, dst, costs, roi_nodes, global_to_roi):
        p, *_ = self.O.dijkstra(self.indptr, self.indices, np.asarray(costs, np.float32), [int(src)], dst=int(dst),
                                roi_map=np.asarray(global_to_roi, np.int32))
        return p.tolist() if len(p) > 1 else None

    def path_to_edges(self, path):
        return self.O.path_to_edges(self.indptr, self.indices, np.asarray(path, np.int32)).tolist()

    def via_penalties(self, st, pres_fac):
        if getattr(st, "via_col_pres", None) is None and getattr(st, "via_seg_pres", None) is None:
            return
        lb = getattr(st, "layer_bias", None)
        self.acct.total_cost = self.O.via_penalties(
            self.acct.total_cost, self.meta, getattr(st, "via_col_pres", None), getattr(st, "via_seg_prefix", None),
            self.nz - 2, lb, pres_fac, st.config.via_column_weight, st.config.via_segment_weight,
            st.config.via_hot_layer_discount)

    def via_block(self, st):
        if getattr(st, "via_col_use", None) is None and getattr(st, "via_seg_use", None) is None:
            return
        self.acct.total_cost = self.O.via_hard_block(
            self.acct.total_cost, self.meta, getattr(st, "via_col_use", None), getattr(st, "via_col_cap", None),
            getattr(st, "via_seg_use", None), getattr(st, "via_seg_cap", None), self.nz - 2)
