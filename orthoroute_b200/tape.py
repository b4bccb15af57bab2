"""Recorded call streams of the reference router ("tapes") and their replay
through the B200 drop-in.

A tape is the ordered list of calls OrthoRoute's PathFinderRouter
(orthoroute/algorithms/manhattan/unified_pathfinder.py, "UPF") made into the
hot path during a real run: the EdgeAccountant methods (UPF:799-1068),
ROIExtractor.extract_roi (UPF:1619), SimpleDijkstra.find_path_roi
(UPF:1801), _path_to_edges (UPF:5463), _apply_via_pooling_penalties
(UPF:3243) and _block_via_edges_with_collisions (UPF:3448), with their
inputs, their outputs (small ones as values, arrays as SHA-1 digests of
their bytes), the reference's time per call, and the writes the loop made to
the accountant's arrays between calls (sparse diffs).  ``replay`` drives any
object set with those methods through a tape and compares every output and
every accountant digest with the recorded one; with the drop-in objects
(orthoroute_b200.dropin.DropInSet) it checks and times the B200 path under
the reference's own call stream without the reference being present.
Tapes are self-contained .npz files (tests/golden/golden_dropin_tape.npz).
"""
from __future__ import annotations

import hashlib
import json
import time
from types import SimpleNamespace

import numpy as np

ACCT_ARRAYS = ("present", "present_ema", "history", "capacity", "total_cost")


def digest(a) -> str:
    """SHA-1 (16 hex digits) of an array's bytes (float32 as bit patterns);
    'none' for None."""
    if a is None:
        return "none"
    a = np.ascontiguousarray(a)
    return hashlib.sha1(a.tobytes()).hexdigest()[:16] + f"_{a.dtype.str}_{a.size}"


class Tape:
    """Events (JSON-able dicts) plus array blobs keyed by digest."""

    def __init__(self, events=None, blobs=None, meta=None):
        self.events = events if events is not None else []
        self.blobs = blobs if blobs is not None else {}
        self.meta = meta if meta is not None else {}

    def blob(self, arr, dtype=None) -> str:
        a = np.ascontiguousarray(arr if dtype is None else np.asarray(arr, dtype=dtype))
        key = digest(a)
        self.blobs.setdefault(key, a.copy())
        return key

    def get(self, key):
        return None if key is None else self.blobs[key]

    def save(self, path):
        arrays = {f"b{i}": v for i, v in enumerate(self.blobs.values())}
        keys = list(self.blobs.keys())
        np.savez_compressed(path, events=np.frombuffer(json.dumps(self.events).encode(), dtype=np.uint8),
                            meta=np.frombuffer(json.dumps(self.meta).encode(), dtype=np.uint8),
                            keys=np.frombuffer(json.dumps(keys).encode(), dtype=np.uint8), **arrays)

    @classmethod
    def load(cls, path) -> "Tape":
        z = np.load(path)
        keys = json.loads(bytes(z["keys"]).decode())
        blobs = {k: z[f"b{i}"] for i, k in enumerate(keys)}
        return cls(json.loads(bytes(z["events"]).decode()), blobs, json.loads(bytes(z["meta"]).decode()))


# ----------------------------------------------------------------------------
# replay

def router_state(tape: Tape, ev: dict, cfg_keys=("col_w", "seg_w", "hot")):
    """The router attributes a via event read, as a namespace (the shape the
    drop-in's via functions take)."""
    st = SimpleNamespace(**{k: tape.get(v) for k, v in ev["state"].items()})
    st._via_edge_metadata = True if ev.get("has_meta") else None
    st.config = SimpleNamespace(via_column_weight=ev.get("col_w", 1.0), via_segment_weight=ev.get("seg_w", 1.0),
                                via_hot_layer_discount=ev.get("hot", 0.20))
    return st


def _dec(tape: Tape, v):
    if isinstance(v, dict) and "blob" in v:
        return tape.get(v["blob"])
    if isinstance(v, list):
        return [_dec(tape, x) for x in v]
    return v


class ReplayReport:
    def __init__(self):
        self.failures = []      # (event index, description)
        self.calls = {}         # kind -> count
        self.searches = 0
        self.paths_equal_reference = 0
        self.paths_equal_oracle = 0
        self.reference_differs = 0   # searches where the reference's float64 path differs from the fp32 oracle's
        self.seconds = {}       # kind -> backend seconds
        self.ref_seconds = {}   # kind -> reference seconds (recorded)

    def fail(self, i, msg):
        self.failures.append((i, msg))

    def add_time(self, kind, sec, ref_sec):
        self.seconds[kind] = self.seconds.get(kind, 0.0) + sec
        self.ref_seconds[kind] = self.ref_seconds.get(kind, 0.0) + (ref_sec or 0.0)
        self.calls[kind] = self.calls.get(kind, 0) + 1


def replay(tape: Tape, backend, *, stop_on_failure: bool = True, timer=time.perf_counter,
           sync=lambda: None) -> ReplayReport:
    """Drives `backend` through the tape.  The backend provides:
      acct                         an EdgeAccountant-like object (host arrays)
      extract_roi(src, dst, initial_radius, stagnation_bonus, portal_seeds) -> (roi, g2r)
      find_path_roi(src, dst, costs, roi_nodes, global_to_roi) -> path or None
      path_to_edges(path) -> edges
      via_penalties(state, pres_fac), via_block(state)   (state: router_state())
    `sync` is called before each timer read (a device synchronisation)."""
    rep = ReplayReport()
    acct = backend.acct
    N = int(tape.meta["N"])
    last_roi = None
    last_path = None
    for i, ev in enumerate(tape.events):
        k = ev["k"]
        if k == "set":
            getattr(acct, ev["name"])[tape.get(ev["idx"])] = tape.get(ev["val"])
            continue
        if k == "full":
            setattr(acct, ev["name"], tape.get(ev["val"]).copy())
            continue
        if k == "canon":
            acct.canonical = {int(a): int(b) for a, b in zip(tape.get(ev["keys"]), tape.get(ev["vals"]))}
            continue
        if k == "iter":
            continue
        sync()
        t0 = timer()
        if k == "acct":
            args = {a: _dec(tape, v) for a, v in ev["args"].items()}
            m = ev["m"]
            if m == "compute_overuse":
                ri = args.pop("router_instance")
                args["router_instance"] = None if ri is None else SimpleNamespace(
                    **{n: tape.get(b) for n, b in ri.items()})
            if m in ("commit_path", "clear_path"):
                args["edge_indices"] = [int(x) for x in args["edge_indices"]]
            out = getattr(acct, m)(**args)
            sync()
            rep.add_time(f"acct.{m}", timer() - t0, ev.get("sec"))
            want = ev["out"]
            got = list(out) if isinstance(out, tuple) else out
            if want != got:
                rep.fail(i, f"{m} returned {got}, the reference {want}")
        elif k == "roi":
            seeds = ev["portal_seeds"]
            roi, g2r = backend.extract_roi(ev["src"], ev["dst"], ev["initial_radius"], ev["stagnation_bonus"],
                                           [tuple(s) for s in seeds] if seeds else None)
            sync()
            rep.add_time("extract_roi", timer() - t0, ev.get("sec"))
            last_roi = roi
            if digest(np.asarray(roi, dtype=np.int32)) != ev["roi"]:
                rep.fail(i, f"ROI of {ev['src']}->{ev['dst']} differs ({len(roi)} nodes, reference {ev['len']})")
        elif k == "search":
            costs = acct.total_cost if ev["costs"] == "total" else _dec(tape, ev["costs"])
            if ev["roi"] == "last":
                roi = last_roi
            elif ev["roi"] == "full":
                roi = np.arange(N, dtype=np.int32)
            else:
                roi = _dec(tape, ev["roi"])
            # the caller's map, built as _route_all builds it (UPF:4690-4692)
            g2r = np.full(N, -1, dtype=np.int32)
            g2r[np.asarray(roi)] = np.arange(len(roi), dtype=np.int32)
            t0 = timer()
            p = backend.find_path_roi(ev["src"], ev["dst"], costs, roi, g2r)
            sync()
            rep.add_time("find_path_roi", timer() - t0, ev.get("sec"))
            got = [int(x) for x in p] if p else None
            rep.searches += 1
            want_oracle = ev.get("oracle", ev["out"])
            if "oracle" in ev:
                rep.reference_differs += 1
            rep.paths_equal_reference += int(got == ev["out"])
            rep.paths_equal_oracle += int(got == want_oracle)
            if got != want_oracle:
                rep.fail(i, f"path {ev['src']}->{ev['dst']} differs from the fp32 oracle's")
            last_path = ev["out"]
        elif k == "p2e":
            path = last_path if ev["path"] == "last" else ev["path"]
            out = backend.path_to_edges(path)
            sync()
            rep.add_time("path_to_edges", timer() - t0, ev.get("sec"))
            if [int(e) for e in out] != ev["out"]:
                rep.fail(i, "path -> edges differs")
        elif k == "via_pen":
            backend.via_penalties(router_state(tape, ev), ev["pres_fac"])
            sync()
            rep.add_time("via_penalties", timer() - t0, ev.get("sec"))
        elif k == "via_block":
            backend.via_block(router_state(tape, ev))
            sync()
            rep.add_time("via_hard_block", timer() - t0, ev.get("sec"))
        else:
            raise ValueError(f"unknown tape event {k}")
        if "after" in ev:
            for name, want in ev["after"].items():
                v = getattr(acct, name, None)
                got = digest(None if v is None else np.asarray(v, dtype=np.float32))
                if got != want:
                    rep.fail(i, f"accounting.{name} after {ev.get('m', k)} differs from the reference's")
        if rep.failures and stop_on_failure:
            break
    return rep


