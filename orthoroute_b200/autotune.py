"""Autotuner for batched box-ROI searches (orsp_sssp_batch_bbox).

The batch kernel has two implementations and a few knobs:

* one CTA per search (block-local near-far): bucket width delta, CTAs per SM;
* tile sweeps over many boxes per launch, each box with its own distance
  slice: tile width 16 or 32.

Which is fastest depends on the ROI size and on the mix: small boxes fit a
CTA's shared memory and finish in a few rounds, large boxes need many SMs,
and all one-CTA searches of a call share one launch, so sizes overlap on the
GPU.  The tuner buckets the searches by node count, tunes the CTA kernel's
parameters per bucket, then times whole plans on a sample of the workload
with CUDA events, checks that every candidate returns the same paths (the
plan may only change the time), and installs the fastest plan on the graph
(orsp_batch_set_plan).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np
import torch

from .solver import DeviceGraph

DEFAULT_EDGES = (4096, 32768, 262144)  # bucket upper bounds (nodes); the last bucket is open


@dataclass
class TuneResult:
    plan: List[dict]
    table: List[Dict[str, float]] = field(default_factory=list)  # per bucket: candidate -> ms per search
    samples: List[int] = field(default_factory=list)


def _candidates(mean_cost: float, is_lattice: bool) -> List[dict]:
    out = []
    for scale in (0.5, 1.0, 2.0, 4.0):
        for ctas in (1, 2):
            out.append({"impl": 0, "delta": float(scale * mean_cost), "ctas_per_sm": ctas, "tile_w": 16})
    if is_lattice:
        for tw in (16, 32):
            out.append({"impl": 1, "delta": 0.0, "ctas_per_sm": 0, "tile_w": tw})
    return out


def _name(c: dict) -> str:
    if c["impl"] == 1:
        return f"sweeps/tile{c['tile_w']}"
    return f"cta/delta{c['delta']:.3g}/x{c['ctas_per_sm']}"


def _time_plan(dg, plan, cost, s, d, b, path_cap, reps):
    dg.set_batch_plan(plan)
    out = dg.batch_bbox(cost, s, d, b, path_cap=path_cap, with_edges=False)  # warm-up
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        dg.batch_bbox(cost, s, d, b, path_cap=path_cap, with_edges=False)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, out


def _same(ref, got, n):
    lr, nr = ref[2].cpu().numpy(), ref[0].cpu().numpy()
    lg, ng = got[2].cpu().numpy(), got[0].cpu().numpy()
    return np.array_equal(lr, lg) and all(np.array_equal(nr[k, : lr[k]], ng[k, : lg[k]]) for k in range(n))


def tune_batch(dg: DeviceGraph, cost: torch.Tensor, src: torch.Tensor, dst: torch.Tensor, boxes: np.ndarray,
               edges: Sequence[int] = DEFAULT_EDGES, sample: int = 1024, bucket_sample: int = 64,
               path_cap: int = 4096, reps: int = 2, seed: int = 0, install: bool = True) -> TuneResult:
    """Tunes the batch plan for a workload like the given searches.

    Stage 1, per ROI-size bucket: the one-CTA-per-search kernel's bucket width
    and CTAs per SM, timed on up to `bucket_sample` searches of the bucket.
    Stage 2, whole plans on a sample of `sample` searches drawn from the whole
    workload (so that buckets share the GPU as they do in the real run): every
    bucket on one CTA per search, or the buckets from a size threshold up on
    tile sweeps (tile width 16 or 32).  Every candidate must return the same
    paths as the first.  boxes: host int32[K, 6]; src/dst/cost: device
    tensors.  Installs the fastest plan on `dg` unless install=False."""
    boxes = np.ascontiguousarray(boxes, dtype=np.int32)
    K = len(boxes)
    vol = (boxes[:, 1] - boxes[:, 0] + 1).astype(np.int64) * (boxes[:, 3] - boxes[:, 2] + 1) * \
        (boxes[:, 5] - boxes[:, 4] + 1)
    bounds = list(edges) + [1 << 40]
    fin = cost[torch.isfinite(cost)]
    mean_cost = float(fin[:: max(1, fin.numel() // 65536)].mean()) if fin.numel() else 1.0
    rng = np.random.default_rng(seed)
    result = TuneResult(plan=[])
    prev = 0
    cta_best: List[dict] = []
    # ---- stage 1: kernel parameters of the one-CTA-per-search implementation
    for ub in bounds:
        idx = np.nonzero((vol > prev) & (vol <= ub))[0]
        prev = ub
        cands = [c for c in _candidates(mean_cost, False)]
        if idx.size == 0:
            cta_best.append(cands[0])
            result.table.append({})
            result.samples.append(0)
            continue
        pick = np.sort(rng.choice(idx, size=min(bucket_sample, idx.size), replace=False))
        pt = torch.from_numpy(pick).to(src.device)
        s, d = src[pt].contiguous(), dst[pt].contiguous()
        b = torch.from_numpy(boxes[pick]).to(src.device)
        times: Dict[str, float] = {}
        ref = None
        best, best_ms = None, float("inf")
        for c in cands:
            ms, out = _time_plan(dg, [{"max_nodes": 1 << 40, **c}], cost, s, d, b, path_cap, reps)
            if ref is None:
                ref = out
            elif not _same(ref, out, len(pick)):
                raise RuntimeError(f"batch plan {_name(c)} changed the paths")
            times[_name(c)] = ms / len(pick)
            if ms < best_ms:
                best, best_ms = c, ms
        cta_best.append(best)
        result.table.append(times)
        result.samples.append(int(len(pick)))
    # ---- stage 2: whole plans on a sample of the workload
    pick = np.sort(rng.choice(K, size=min(sample, K), replace=False))
    pt = torch.from_numpy(pick).to(src.device)
    s, d = src[pt].contiguous(), dst[pt].contiguous()
    b = torch.from_numpy(boxes[pick]).to(src.device)
    plans = {"default": None, "cta": [{"max_nodes": int(ub), **c} for ub, c in zip(bounds, cta_best)]}
    if getattr(dg, "lattice_kind", int(dg.is_lattice)) == 1:  # batched tile sweeps need adjacent-layer vias
        for cut in range(len(bounds)):
            for tw in (16, 32):
                plans[f"sweeps>={cut}/tile{tw}"] = [
                    {"max_nodes": int(ub), **(c if i < cut else {"impl": 1, "delta": 0.0, "ctas_per_sm": 0,
                                                                  "tile_w": tw})}
                    for i, (ub, c) in enumerate(zip(bounds, cta_best))]
    ref = None
    best_plan, best_ms = None, float("inf")
    whole: Dict[str, float] = {}
    for name, plan in plans.items():
        ms, out = _time_plan(dg, plan, cost, s, d, b, path_cap, reps)
        if ref is None:
            ref = out
        elif not _same(ref, out, len(pick)):
            raise RuntimeError(f"batch plan {name} changed the paths")
        whole[name] = ms / len(pick)
        if ms < best_ms:
            best_plan, best_ms = plan, ms
    result.plan.extend(best_plan or [])
    result.table.append({"whole:" + k: v for k, v in whole.items()})
    result.samples.append(int(len(pick)))
    if install:
        dg.set_batch_plan(best_plan)
    else:
        dg.set_batch_plan(getattr(dg, "batch_plan", None))
    return result
