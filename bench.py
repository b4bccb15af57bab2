#!/usr/bin/env python
"""Benchmark of the PathFinder SSSP hot path on one or more B200s.

Workload (one "step"): the single-source SSSP sweep on the 1000x1000x12
alternating-H/V lattice with adjacent-layer vias (12.0 M nodes, 45.98 M
directed edges, int32 CSR), fp32 weights uniform in [1,2) on planar edges,
3.0 on vias, 5 % of edges blocked (+inf), seeded; 64 random sources as full
searches over the whole grid, 16 sources per tile-search launch
(orsp_sssp_sources, --per-launch; 0 runs them one at a time).  The
one-source-at-a-time sweep is timed beside it ("single_search").  Every
source's distances are checked bit for bit against the CPU oracle before
timing, from both modes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is GTEPS over the timed steps with
inputs resident in HBM; `e2e` repeats the sweep through the public API with
the weights copied from pinned host memory and every distance array copied
back each step.  With N > 1 (torchrun) every rank runs its own replica of the
workload (different seeds) - the search does not shard - and the times are the
max over ranks.

The `routing` object reports seconds to a zero-overuse route on two boards
(100x100x4 with 200 nets; the 600x600x18 backplane with 8 000 nets, one GPU
only), plain vs batched, with the routes checked identical; --no-route skips
it.  The `batch_sweep` object reports the batched uneven-ROI sweep (4 096 box
searches, one GPU only): one search per launch vs the default and the tuned
batch plan; --no-sweep skips it.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "sec to zero-overuse route, batched+warm vs plain, 1 B200; SSSP GTEPS & HBM GB/s"
NX, NY, NZ = 1000, 1000, 12
NSRC = 64
PER_LAUNCH = 16
# backplane board (route_c3), batched + warm: nets per snapshot group and
# repair rounds (orsp_route_nets_snapshot)
C3_GROUP, C3_REPAIR = 32, 3
BLOCKED = 0.05
SEED = 20261203
# DRAM bytes (read + write) per lattice node and source of the tile search in
# a many-source launch (lattice_spec_kernel, two CTAs per SM), from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on a 4-source launch of the
# 1000x1000x12 lattice (bench.py --profile-case --per-launch 4), with the
# scheduler warp's L2 prefetch: 971.27 + 178.85 MB for 4 x 12.0 M
# node-sources.  Every search settles every node;
# the traffic is the distance slices read and written about once plus the
# shared weights, so it grows with the sources per launch.
LAT_DRAM_BYTES_PER_NODE = (971.270912e6 + 178.853888e6) / (4 * 1000 * 1000 * 12)


def _peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class NvmlClockSampler:
    """SM clock, its maximum and the clock-event (throttle) reasons of one
    GPU, read through NVML every 10 ms from a thread while the timed region
    runs, plus one reading at start and one at stop (a region of a few
    hundred ms still gets samples).  Only reads the GPU's state."""

    REASONS = (("hw_slowdown", "HwSlowdown"), ("hw_thermal_slowdown", "HwThermalSlowdown"),
               ("sw_thermal_slowdown", "SwThermalSlowdown"), ("sw_power_cap", "SwPowerCap"))

    def __init__(self, device):
        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        props = __import__("torch").cuda.get_device_properties(device)
        h = None
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
        except Exception:
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(
                    "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id))
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(int(getattr(device, "index", 0) or 0))
        self.h = h
        self.bits = {name: getattr(pynvml, "nvmlClocksEventReason" + key,
                                   getattr(pynvml, "nvmlClocksThrottleReason" + key, 0)) for name, key in self.REASONS}
        self.reasons_fn = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        self.rows = []
        self.stop_flag = None
        self.thread = None

    def _read(self):
        nv = self.nv
        self.rows.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                          nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM), int(self.reasons_fn(self.h))))

    def start(self):
        import threading

        self.stop_flag = threading.Event()
        self._read()

        def loop():
            while not self.stop_flag.wait(0.01):
                try:
                    self._read()
                except Exception:
                    return

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        self.stop_flag.set()
        self.thread.join(timeout=5)
        self._read()
        sm = [float(r[0]) for r in self.rows]
        load = [v for v in sm if v > 0.5 * max(sm)] if sm else []
        reasons = sorted({name for r in self.rows for name, bit in self.bits.items() if bit and (r[2] & bit)})
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(float(r[1]) for r in self.rows) if self.rows else None,
                "reasons": reasons, "samples": len(self.rows), "sampler": "nvml, 10 ms"}


def clock_sampler(device):
    """The NVML sampler, else nvidia-smi's (200 ms)."""
    try:
        return NvmlClockSampler(device)
    except Exception:
        return ClockSampler(getattr(device, "index", 0) or 0)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def workload_config(args, lat, nsrc: int, world: int) -> dict:
    """The workload description both arms print (the same keys and values)."""
    return {"workload": f"sssp_{args.nx}x{args.ny}x{args.nz}_{nsrc}src_full", "nodes": lat.N, "edges": lat.E,
            "sources_per_step": nsrc, "weights": "fp32 uniform [1,2) planar, 3.0 via, 5% +inf",
            "l2": "inputs larger than L2 (CSR + weights + distances ~0.6 GB)", "parallelism": f"replicas x{world}"}


def make_workload(seed: int, nx=NX, ny=NY, nz=NZ, nsrc=NSRC):
    from orthoroute_b200.lattice import build_lattice, uniform_weights

    lat = build_lattice(nx, ny, nz)
    w = uniform_weights(lat, seed=seed, blocked_frac=BLOCKED)
    rng = np.random.default_rng(seed + 1)
    sources = rng.choice(lat.N, size=nsrc, replace=False).astype(np.int32)
    return lat, w, sources


def cpu_baseline(lat, w, sources, threads: int, budget_s: float = 20.0):
    """The oracle (C heap Dijkstra, one source per thread, ctypes releases the
    GIL) on a bounded sample of the same workload."""
    import oracle as O
    from concurrent.futures import ThreadPoolExecutor

    O.build_oracle()
    deg = np.diff(lat.indptr)

    def one(s):
        _, dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(s)])
        return int(deg[np.isfinite(dist)].sum())

    sample = list(sources[:threads])
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        edges = sum(ex.map(one, sample))
    t = time.perf_counter() - t0
    return {"value": edges / t / 1e9, "unit": "GTEPS", "cores": threads, "kind": "port",
            "sample": f"{len(sample)} full single-source searches of the same lattice in parallel "
                      f"({t:.1f} s wall)"}


def parity_all_sources(dg, wt, lat, w, sources, threads: int, per_launch: int = 0):
    """Every source's distances against the C oracle, bit for bit (the oracle
    runs one source per host thread while the GPU computes the next), from
    the one-source search and, with per_launch > 0, from the many-source
    launch (orsp_sssp_sources) as well."""
    import torch

    import oracle as O
    from concurrent.futures import ThreadPoolExecutor

    O.build_oracle()
    dist = torch.empty(lat.N, dtype=torch.float32, device=wt.device)
    ok = True
    t0 = time.perf_counter()

    def ref(s):
        return O.dijkstra(lat.indptr, lat.indices, w, [int(s)])[1].view(np.uint32)

    rows = None
    if per_launch > 0:
        rows = torch.empty(len(sources), lat.N, dtype=torch.float32, device=wt.device)
        for a in range(0, len(sources), per_launch):
            dg.sssp_sources(wt, sources[a:a + per_launch], rows[a:a + per_launch], per_launch=per_launch)
    with ThreadPoolExecutor(max_workers=threads) as ex:
        for b0 in range(0, len(sources), threads):
            batch = sources[b0:b0 + threads]
            futs = [ex.submit(ref, s) for s in batch]
            for i, (s, f) in enumerate(zip(batch, futs)):
                dg.sssp(wt, int(s), -1, dist_out=dist)
                got = dist.cpu().numpy().view(np.uint32)
                want = f.result()
                ok = ok and bool(np.array_equal(got, want))
                if rows is not None:
                    ok = ok and bool(np.array_equal(rows[b0 + i].cpu().numpy().view(np.uint32), want))
    return {"sources_checked": len(sources), "identical_to_oracle": ok,
            "paths_checked": "one-source searches" + (f" and {per_launch}-source launches" if rows is not None else ""),
            "oracle": f"C heap Dijkstra (fp32), {threads} host threads, {time.perf_counter() - t0:.1f} s"}


def route_dropin(dev, with_cpu: bool):
    """The reference router's own call stream into the hot path, replayed
    through the drop-in (orthoroute_b200.dropin.DropInSet): the tape of the
    unmodified PathFinderRouter routing the 100x100x4 board with 200 nets for
    three iterations (tests/golden/golden_dropin_tape.npz; accountant
    updates, ROI extractions, searches, path -> edges, via steps).  Every
    result is compared with the tape; per-call latency is reported against
    the reference's own time for the same calls (recorded single-threaded
    when the tape was made) and the C oracle's on this host."""
    import torch

    from orthoroute_b200.dropin import DropInSet
    from orthoroute_b200.lattice import build_lattice
    from orthoroute_b200.tape import Tape, replay

    tape = Tape.load(REPO / "tests" / "golden" / "golden_dropin_tape.npz")
    m = tape.meta
    lat = build_lattice(m["nx"], m["ny"], m["nz"])

    def run():
        ds = DropInSet(lat.indptr, lat.indices, lattice=lat, nx=lat.nx, ny=lat.ny, nz=lat.nz, device=dev)
        return replay(tape, ds, sync=lambda: torch.cuda.synchronize(dev))

    run()  # warm-up: library workspaces and first-call set-up
    rep = run()
    out = {
        "workload": "reference PathFinderRouter call stream: " + m["board"] + f", iterations 1-{m['iterations']}",
        "identical_to_reference_tape": not rep.failures,
        "searches": rep.searches,
        "paths_equal_reference": rep.paths_equal_reference,
        "paths_equal_fp32_oracle": rep.paths_equal_oracle,
        "calls": {},
    }
    hot = 0.0
    hot_ref = 0.0
    for kind, n in sorted(rep.calls.items()):
        ours = rep.seconds[kind] / n
        ref = rep.ref_seconds[kind] / n
        hot += rep.seconds[kind]
        hot_ref += rep.ref_seconds[kind]
        out["calls"][kind] = {"n": n, "us_per_call": round(ours * 1e6, 1),
                              "reference_us_per_call": round(ref * 1e6, 1),
                              "speedup": round(ref / ours, 1) if ours > 0 else None}
    out["sec_total"] = round(hot, 4)
    out["reference_sec_total"] = round(hot_ref, 3)
    out["speedup_vs_reference"] = round(hot_ref / hot, 1) if hot > 0 else None
    out["reference_timing"] = "the unmodified reference (Python, 1 core) timed per call when the tape was recorded"
    if with_cpu:
        import oracle as O
        from oracle.dropin_tape import OracleBackend

        O.build_oracle()
        be = OracleBackend(lat.indptr, lat.indices, lat.nx, lat.ny, lat.nz)
        ro = replay(tape, be)
        out["cpu_oracle_sec_total"] = round(sum(ro.seconds.values()), 3)
        out["cpu_oracle_identical"] = not ro.failures
        out["cpu_oracle_cores"] = 1
    return out


def roi_searches(dev, nsamp: int = 48, ncheck: int = 8):
    """BFS-ROI searches as the reference's _route_all issues them: for net
    (s, d), find_path_roi over extract_roi_bfs(s, d) with depth min(max(60,
    0.75 * manhattan), 150) and at most 50 000 nodes (UPF:1619-1734,
    4614-4785), on the config-1 board (100x100x4, 200 nets) and the config-3
    board (600x600x18, 8 000 nets), nsamp nets each, fp32 costs uniform in
    [1, 2) with vias at 3.  Per search (the synchronous C-ABI call, ROI
    already on the device): the tile-sweep ROI search against the generic
    grid kernel it replaced ("before").  On the same boards built as the
    reference's own Lattice3D graph (inner-layer planar edges, vias between
    any two layers, duplicated via edges): the tile sweeps with the column
    via pass (the graph given its dimensions), against the one-CTA search and
    the grid kernel (the same CSR without dimensions).  Paths must agree
    across implementations and with the oracle on ncheck nets."""
    import torch

    import oracle as O
    from orthoroute_b200 import _lib
    from orthoroute_b200.lattice import board_footprints, board_uniform_pins, build_lattice, uniform_weights
    from orthoroute_b200.solver import DeviceGraph

    O.build_oracle()
    out = {}
    keys = ("ORSP_SSSP_IMPL", "ORSP_ROI_NODES_IMPL")
    saved = {k: os.environ.get(k) for k in keys}
    try:
        for name, (nx, ny, nz), make in (
                ("c1", (100, 100, 4), lambda: board_uniform_pins(100, 100, 4, 200, seed=1)),
                ("c3", (600, 600, 18), lambda: board_footprints(600, 600, 18, 8000, None, seed=3))):
            b = make()
            rng = np.random.default_rng(5)
            pick = rng.choice(len(b.src), size=min(nsamp, len(b.src)), replace=False)
            nets = [(int(b.src[i]), int(b.dst[i])) for i in pick]
            row = {}
            for shape, lat in (("lattice", b.lattice),
                               ("reference_lattice3d", build_lattice(nx, ny, nz, planar="inner", vias="full",
                                                                     duplicate_vias=True))):
                w = uniform_weights(lat, seed=11)
                wt = torch.from_numpy(w).to(dev)
                dg = DeviceGraph.from_lattice(lat, device=dev)  # tile lattice, or column vias
                flat = None if shape == "lattice" else DeviceGraph(lat.indptr, lat.indices, device=dev)
                rois = []
                for s_, d_ in nets:
                    (sx, sy, _), (dx, dy, _) = lat.coords(s_), lat.coords(d_)
                    depth = min(max(60, int(0.75 * (abs(int(dx) - int(sx)) + abs(int(dy) - int(sy))))), 150)
                    roi, _ = dg.roi_bfs(s_, d_, depth, 50_000, want_g2r=False)
                    rois.append(roi.clone())
                impls = ({"tile_sweeps": ({"ORSP_SSSP_IMPL": "auto"}, dg),
                          "grid_before": ({"ORSP_SSSP_IMPL": "generic", "ORSP_ROI_NODES_IMPL": "grid"}, dg)}
                         if shape == "lattice" else
                         {"tile_sweeps_column_vias": ({"ORSP_SSSP_IMPL": "auto"}, dg),
                          "one_cta": ({"ORSP_ROI_NODES_IMPL": "cta"}, flat),
                          "grid_before": ({"ORSP_ROI_NODES_IMPL": "grid"}, flat)})
                res, paths = {}, {}
                for iname, (env, gr) in impls.items():
                    for k in keys:
                        os.environ.pop(k, None)
                    os.environ.update(env)
                    for (s_, d_), roi in list(zip(nets, rois))[:4]:  # warm-up
                        gr.sssp_roi_nodes(wt, s_, d_, roi)
                    torch.cuda.synchronize(dev)
                    got = []
                    t0 = time.perf_counter()
                    for (s_, d_), roi in zip(nets, rois):
                        st, pth = gr.sssp_roi_nodes(wt, s_, d_, roi)
                        got.append(pth.cpu().numpy().copy() if st == _lib.ORSP_OK else None)
                    dt = time.perf_counter() - t0
                    res[iname] = {"ms_per_search": round(dt / len(nets) * 1e3, 3)}
                    paths[iname] = got
                names = list(impls)
                same = all(all((a is None and c is None) or (a is not None and c is not None and np.array_equal(a, c))
                               for a, c in zip(paths[names[0]], paths[nm])) for nm in names[1:])
                ok = True
                for (s_, d_), roi, pth in list(zip(nets, rois, paths[names[0]]))[:ncheck]:
                    r = roi.cpu().numpy()
                    g2r = np.full(lat.N, -1, np.int32)
                    g2r[r] = np.arange(len(r), dtype=np.int32)
                    ref, *_ = O.dijkstra(lat.indptr, lat.indices, w, [s_], dst=d_, roi_map=g2r)
                    want = ref if len(ref) > 1 else None
                    ok = ok and ((pth is None and want is None) or
                                 (pth is not None and want is not None and np.array_equal(pth, want)))
                res["speedup_vs_grid"] = round(res["grid_before"]["ms_per_search"] / res[names[0]]["ms_per_search"], 2)
                res["mean_roi_nodes"] = int(np.mean([len(r) for r in rois]))
                res["identical_paths"] = bool(same)
                res["identical_to_oracle"] = bool(ok)
                row[shape] = res
                dg.close()
                if flat is not None:
                    flat.close()
            out[name] = row
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    out["workload"] = (f"{nsamp} BFS-ROI searches per board (reference radius rule, <= 50 000 nodes), "
                       f"synchronous calls; oracle checked on {ncheck}")
    return out


def route_c1(dev, with_cpu: bool):
    """The 100x100x4 board (200 two-pin nets, pins uniform on the top
    layer, seeded) routed to zero overuse with per-net live costs, offenders
    rerouted after iteration 1: plain (one search per net) vs batched (one
    launch per level of disjoint boxes).  Identical routes by construction
    (and checked by tests/test_gpu_negotiation.py)."""
    import torch

    from orthoroute_b200.lattice import board_uniform_pins
    from orthoroute_b200.negotiate import NegotiationConfig, PathFinder

    b = board_uniform_pins(100, 100, 4, 200, seed=1)
    cfg = NegotiationConfig(cost_update="net", reroute="offenders", full_graph_retry=False)
    pf = PathFinder(b.lattice, config=cfg, device=dev)
    pf.route(b.src, b.dst, mode="batched")  # warm-up (graph upload, workspaces)
    rb = pf.route(b.src, b.dst, mode="batched")
    rs = pf.route(b.src, b.dst, mode="sequential")
    same = rb.overuse_trace() == rs.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(rb.paths, rs.paths))
    # the oracle loop (C heap Dijkstra, numpy accounting) on the same board
    import oracle as O
    from oracle.negotiate import route_plain

    O.build_oracle()
    ref = route_plain(b.lattice, b.src, b.dst, cfg)
    out_same = [(s_, c_) for s_, c_, _ in ref["trace"]] == rb.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(rb.paths, ref["paths"])) and np.array_equal(rb.edge_usage, ref["usage"])
    # snapshot groups (the config-3 warm run's schedule) from zero history,
    # against the oracle loop of the same schedule
    import dataclasses

    cfg_s = dataclasses.replace(cfg, net_order="disjoint", group_nets=C3_GROUP, group_repair=C3_REPAIR)
    pf.cfg = cfg_s
    pf.route(b.src, b.dst, mode="batched")  # warm-up of the snapshot workspaces
    rg = pf.route(b.src, b.dst, mode="batched")
    pf.cfg = cfg
    ref_s = route_plain(b.lattice, b.src, b.dst, cfg_s)
    snap_same = [(s_, c_) for s_, c_, _ in ref_s["trace"]] == rg.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(rg.paths, ref_s["paths"])) and np.array_equal(rg.edge_usage,
                                                                                         ref_s["usage"])
    out = {
        "workload": "100x100x4 lattice, 200 two-pin nets, per-net live costs, offenders rerouted",
        "identical_to_oracle": bool(out_same and same),
        "converged": bool(rb.converged),
        "iterations": len(rb.iterations),
        "sec_batched": round(rb.seconds, 4),
        "sec_plain": round(rs.seconds, 4),
        "speedup_batched_vs_plain": round(rs.seconds / rb.seconds, 2),
        "identical_routes": bool(same),
        "wirelength": rb.wirelength,
        "vias": rb.vias,
        "overuse_trace": [s.over_sum for s in rb.iterations],
        "snapshot": {"schedule": f"snapshot groups of {C3_GROUP} nets in the disjoint-round order, {C3_REPAIR} "
                                 "repair rounds, zero history",
                     "identical_to_oracle": bool(snap_same), "converged": bool(rg.converged),
                     "iterations": len(rg.iterations), "sec": round(rg.seconds, 4),
                     "speedup_vs_plain": round(rs.seconds / rg.seconds, 2),
                     "wirelength_delta_pct": round(100.0 * (rg.wirelength - rb.wirelength) / max(1, rb.wirelength), 3),
                     "vias_delta_pct": round(100.0 * (rg.vias - rb.vias) / max(1, rb.vias), 3)},
    }
    if with_cpu:
        out["cpu_oracle_sec"] = round(ref["seconds"], 3)
        out["cpu_oracle_iterations"] = len(ref["trace"])
        out["cpu_oracle_cores"] = 1
    return out


def route_c3(dev, with_cpu: bool):
    """Backplane board (600x600x18 lattice, 8 000 two-pin nets between 2x50-pin
    connector footprints, one net per pin, ROI = bounding box + 10 cells)
    routed to zero overuse with per-net live costs: plain (one search launch
    per net, the device loop orsp_route_nets) vs batched (one launch per round
    of pairwise disjoint boxes).  Both take the nets in the same first-fit
    disjoint-round order and widen the box of a net that offends twice
    running by 10 cells, so their routes are identical (checked here).
    Batched + warm: the learned history prior and snapshot groups of
    C3_GROUP nets (orsp_route_nets_snapshot: one launch per group on one
    cost snapshot, then C3_REPAIR repair rounds), a schedule of its own whose
    wirelength and vias are reported against the plain routes."""
    from orthoroute_b200.lattice import board_footprints
    from orthoroute_b200.negotiate import NegotiationConfig, PathFinder

    import dataclasses

    b = board_footprints(600, 600, 18, 8000, None, seed=3)
    cfg = NegotiationConfig(max_iterations=40, cost_update="net", reroute="offenders", roi_margin=10,
                            full_graph_retry=False, net_order="disjoint", stall_grow=10, stall_iterations=2)
    pf = PathFinder(b.lattice, config=cfg, device=dev)
    # parity at full lattice size: iteration 1 of the first 200 nets, GPU
    # (batched) against the oracle loop, per net and in the final usage
    import oracle as O
    from oracle.negotiate import route_plain

    O.build_oracle()
    sub = 200
    cfg1 = dataclasses.replace(cfg, max_iterations=1)
    pf1 = PathFinder(b.lattice, config=cfg1, device=dev)
    r1 = pf1.route(b.src[:sub], b.dst[:sub], mode="batched")
    t0 = time.perf_counter()
    ref1 = route_plain(b.lattice, b.src[:sub], b.dst[:sub], cfg1)
    t_ref1 = time.perf_counter() - t0
    sub_same = [(s_, c_) for s_, c_, _ in ref1["trace"]] == r1.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(r1.paths, ref1["paths"])) and np.array_equal(r1.edge_usage, ref1["usage"])
    # the same check for the snapshot-group schedule of the warm run, on the
    # first three groups
    sub_s = 3 * C3_GROUP
    cfg1s = dataclasses.replace(cfg1, group_nets=C3_GROUP, group_repair=C3_REPAIR)
    pf1.cfg = cfg1s
    r1s = pf1.route(b.src[:sub_s], b.dst[:sub_s], mode="batched")
    ref1s = route_plain(b.lattice, b.src[:sub_s], b.dst[:sub_s], cfg1s)
    sub_same_snap = [(s_, c_) for s_, c_, _ in ref1s["trace"]] == r1s.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(r1s.paths, ref1s["paths"])) and np.array_equal(r1s.edge_usage,
                                                                                          ref1s["usage"])
    del pf1
    rb = pf.route(b.src, b.dst, mode="batched")
    rs = pf.route(b.src, b.dst, mode="sequential")
    same = rb.overuse_trace() == rs.overuse_trace() and all(
        np.array_equal(x, y) for x, y in zip(rb.paths, rs.paths)) and np.array_equal(rb.edge_usage, rs.edge_usage)
    searches = int(sum(s.nets_searched for s in rb.iterations))
    # batched + learned warm start (orthoroute_b200/data/warm_history.npz):
    # features, inference and the history mapping count in its time; the
    # run gets at most 1.5x the plain iterations, else the plain route is used
    import math

    import torch

    from orthoroute_b200.warm import load_pretrained, warm_history_device

    net, scale = load_pretrained(device=dev)
    # untimed warm-up of the prediction path on a small board (module loads,
    # kernel attributes, allocator); the timed call below does all the work
    # for this board
    wb = board_footprints(64, 64, 18, 80, None, seed=11)
    warm_history_device(net, wb.lattice, wb.src, wb.dst, scale)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    h0 = warm_history_device(net, b.lattice, b.src, b.dst, scale)
    torch.cuda.synchronize(dev)
    t_pred = time.perf_counter() - t0
    # the warm run: snapshot groups of C3_GROUP nets with C3_REPAIR repair
    # rounds (per-net live costs between groups); the same prediction under
    # the exact disjoint-round schedule, and the snapshot schedule from zero
    # history, run beside it
    warm_cfg = dataclasses.replace(cfg, max_iterations=int(math.ceil(1.5 * len(rs.iterations))),
                                   group_nets=C3_GROUP, group_repair=C3_REPAIR)
    pf.cfg = warm_cfg
    rw = pf.route(b.src, b.dst, mode="batched", history_init=h0)
    warm_sec = t_pred + rw.seconds + (0.0 if rw.converged else rb.seconds)
    pf.cfg = dataclasses.replace(warm_cfg, group_nets=0, group_repair=0)
    rwx = pf.route(b.src, b.dst, mode="batched", history_init=h0)
    warm_exact_sec = t_pred + rwx.seconds + (0.0 if rwx.converged else rb.seconds)
    pf.cfg = dataclasses.replace(warm_cfg, max_iterations=cfg.max_iterations)
    rsc = pf.route(b.src, b.dst, mode="batched")
    snap_sec = rsc.seconds + (0.0 if rsc.converged else rb.seconds)
    pf.cfg = cfg

    def _delta(r):
        return {"wirelength_delta_pct": round(100.0 * (r.wirelength - rb.wirelength) / max(1, rb.wirelength), 3),
                "vias_delta_pct": round(100.0 * (r.vias - rb.vias) / max(1, rb.vias), 3)}
    # ablation: the same schedule from a non-learned prior (RUDY wire density,
    # warm.rudy_prediction) at the scale chosen for it on the same held-out
    # boards as the network's
    from orthoroute_b200.warm import history_from_prediction_device, pretrained_rudy_scale, rudy_prediction

    rudy_scale = pretrained_rudy_scale()
    ablation = None
    if rudy_scale is not None:
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        pr = torch.from_numpy(rudy_prediction(b.lattice, b.src, b.dst)).to(dev)
        hr = history_from_prediction_device(b.lattice, pr, rudy_scale)
        torch.cuda.synchronize(dev)
        t_rudy = time.perf_counter() - t0
        pf.cfg = warm_cfg
        ra = pf.route(b.src, b.dst, mode="batched", history_init=hr)
        pf.cfg = cfg
        torch.cuda.synchronize(dev)
        a_sec = t_rudy + ra.seconds + (0.0 if ra.converged else rb.seconds)
        ablation = {"prior": "RUDY (half-perimeter wire length spread over each net's bounding box), not learned",
                    "history_scale": rudy_scale, "sec_batched_prior": round(a_sec, 3),
                    "converged": bool(ra.converged), "iterations": len(ra.iterations),
                    "searches": int(sum(s_.nets_searched for s_ in ra.iterations)),
                    "speedup_vs_plain": round(rs.seconds / a_sec, 2),
                    "wirelength_delta_pct": round(100.0 * (ra.wirelength - rb.wirelength) / max(1, rb.wirelength), 3),
                    "vias_delta_pct": round(100.0 * (ra.vias - rb.vias) / max(1, rb.vias), 3)}
    out = {
        "workload": "600x600x18 lattice, 8000 nets between 2x50 connector footprints, bbox+10 ROI, "
                    "per-net live costs, offenders rerouted, disjoint-round order",
        "footprints": int(b.meta["footprints"]),
        "footprints_note": "176 footprints of 2x50 pins, not 40: 40 x 100 = 4 000 pins cannot give each of the "
                           "16 000 net endpoints its own pin, and a top-layer pin has 3 out-edges of capacity 1",
        "iteration1_subset_identical_to_oracle": bool(sub_same),
        "iteration1_subset": f"first {sub} nets, iteration 1, batched GPU vs the oracle loop "
                             f"({t_ref1:.1f} s on 1 host core)",
        "iteration1_subset_snapshot_identical_to_oracle": bool(sub_same_snap),
        "iteration1_subset_snapshot": f"first {sub_s} nets, iteration 1 of the warm run's snapshot schedule "
                                      f"(zero history), batched GPU vs the oracle loop",
        "converged": bool(rb.converged),
        "iterations": len(rb.iterations),
        "searches": searches,
        "sec_batched": round(rb.seconds, 3),
        "sec_plain": round(rs.seconds, 3),
        "speedup_batched_vs_plain": round(rs.seconds / rb.seconds, 2),
        "identical_routes": bool(same),
        "wirelength": rb.wirelength,
        "vias": rb.vias,
        "overuse_trace": [s.over_sum for s in rb.iterations],
        "warm": {
            "sec_batched_warm": round(warm_sec, 3),
            "sec_prediction": round(t_pred, 3),
            "converged": bool(rw.converged),
            "fell_back_to_plain": not rw.converged,
            "iterations": len(rw.iterations),
            "searches": int(sum(s.nets_searched for s in rw.iterations)),
            "history_scale": scale,
            "schedule": f"snapshot groups of {C3_GROUP} nets in the disjoint-round order, each searched in one "
                        f"launch on the costs after the group's rip-ups, then up to {C3_REPAIR} rounds "
                        "re-searching the nets that share an edge with an earlier net of the group; per-net live "
                        "costs between groups; from the predicted history",
            "speedup_vs_plain": round(rs.seconds / warm_sec, 2),
            "speedup_vs_batched": round(rb.seconds / warm_sec, 2),
            "wirelength": rw.wirelength,
            "vias": rw.vias,
            "wirelength_delta_pct": round(100.0 * (rw.wirelength - rb.wirelength) / max(1, rb.wirelength), 3),
            "vias_delta_pct": round(100.0 * (rw.vias - rb.vias) / max(1, rb.vias), 3),
            "overuse_trace": [s.over_sum for s in rw.iterations],
            "exact_schedule": {"sec": round(warm_exact_sec, 3), "converged": bool(rwx.converged),
                               "iterations": len(rwx.iterations),
                               "searches": int(sum(s.nets_searched for s in rwx.iterations)),
                               "speedup_vs_plain": round(rs.seconds / warm_exact_sec, 2),
                               "note": "the same prediction, one launch per round of disjoint boxes", **_delta(rwx)},
            "snapshot_from_zero_history": {"sec": round(snap_sec, 3), "converged": bool(rsc.converged),
                                           "iterations": len(rsc.iterations),
                                           "searches": int(sum(s.nets_searched for s in rsc.iterations)),
                                           "speedup_vs_plain": round(rs.seconds / snap_sec, 2), **_delta(rsc)},
        },
        "ablation_non_learned_prior": ablation,
    }
    if with_cpu:
        # The C oracle of one box search (heap Dijkstra, fp32) on a sample of
        # iteration-1 nets, scaled to the run's search count: a full CPU run of
        # this board takes hours.
        import oracle as O

        O.build_oracle()
        lat = b.lattice
        from orthoroute_b200.lattice import bbox_with_margin

        boxes = bbox_with_margin(lat, b.src, b.dst, 10)
        sample = np.random.default_rng(0).choice(len(b.src), size=12, replace=False)
        t0 = time.perf_counter()
        for k in sample:
            O.batch_bbox(lat.indptr, lat.indices, lat.base_cost, lat.nx, lat.ny, lat.nz, b.src[k:k + 1],
                         b.dst[k:k + 1], boxes[k:k + 1], 8192)
        per = (time.perf_counter() - t0) / len(sample)
        out["cpu_oracle_sec_per_search"] = round(per, 4)
        out["cpu_oracle_sec_extrapolated"] = round(per * searches, 1)
        out["cpu_oracle_sample"] = f"{len(sample)} iteration-1 box searches, 1 core, scaled to {searches} searches"
    return out


def sweep_c4(dev, nsearch: int = 4096):
    """Batched uneven-ROI sweep: 4 096 independent box searches on one shared
    fp32 cost array (400x400x16 lattice, weights uniform in [1,2), vias 3.0,
    3 % blocked), box sides log-uniform per axis (x, y in [20, 400], z in
    [4, 16]), source and target uniform in each box.  Three runs of the same
    searches: one search per launch (orsp_sssp_box), the default batch plan
    (one CTA per search), and the plan the autotuner picks per ROI-size
    bucket; the paths must be identical."""
    import torch

    from orthoroute_b200.autotune import tune_batch
    from orthoroute_b200.lattice import box_edge_count, build_lattice, random_boxes, uniform_weights
    from orthoroute_b200.solver import DeviceGraph

    lat = build_lattice(400, 400, 16)
    w = uniform_weights(lat, seed=SEED + 4, blocked_frac=0.03)
    boxes, src, dst = random_boxes(lat, nsearch, seed=SEED + 5, lo=(20, 20, 4), hi=(400, 400, 16))
    dg = DeviceGraph.from_lattice(lat, device=dev)
    wt = torch.from_numpy(w).to(dev)
    s_d = torch.from_numpy(src).to(dev)
    t_d = torch.from_numpy(dst).to(dev)
    b_d = torch.from_numpy(boxes).to(dev)
    cap = 4096
    roi_edges = int(box_edge_count(lat, boxes).sum())

    def timed(fn):
        fn()  # warm-up (workspaces)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 1e3, out

    def one_per_launch():
        lens = np.zeros(nsearch, np.int32)
        rows = []
        for k in range(nsearch):
            st, p, _ = dg.sssp_box(wt, int(src[k]), int(dst[k]), boxes[k], path_cap=cap)
            rows.append(p.clone() if p is not None else None)
        return rows

    def batch():
        return dg.batch_bbox(wt, s_d, t_d, b_d, path_cap=cap, with_edges=True)

    t_single, rows = timed(one_per_launch)
    dg.set_batch_plan(None)
    t_default, (n0, _, l0) = timed(batch)
    t0 = time.perf_counter()
    tune = tune_batch(dg, wt, s_d, t_d, boxes, sample=1024, path_cap=cap)
    t_tune = time.perf_counter() - t0
    t_tuned, (n1, _, l1) = timed(batch)
    l0, l1 = l0.cpu().numpy(), l1.cpu().numpy()
    n0, n1 = n0.cpu().numpy(), n1.cpu().numpy()
    same = np.array_equal(l0, l1) and all(np.array_equal(n0[k, : l0[k]], n1[k, : l1[k]]) for k in range(nsearch))
    same_single = all(
        (rows[k] is None and l0[k] < 2) or (rows[k] is not None and l0[k] == rows[k].numel() and
                                              np.array_equal(rows[k].cpu().numpy(), n0[k, : l0[k]]))
        for k in range(nsearch))
    vol = ((boxes[:, 1] - boxes[:, 0] + 1).astype(np.int64) * (boxes[:, 3] - boxes[:, 2] + 1) *
           (boxes[:, 5] - boxes[:, 4] + 1))
    # oracle sample: 64 of the searches, C heap Dijkstra on the same boxes
    import oracle as O

    O.build_oracle()
    pick = np.random.default_rng(SEED + 6).choice(nsearch, size=64, replace=False)
    rn, rl = O.batch_bbox(lat.indptr, lat.indices, w, lat.nx, lat.ny, lat.nz, src[pick], dst[pick], boxes[pick], cap)
    same_oracle = all(
        (l1[k] < 2 and rl[j] < 2) or (l1[k] == rl[j] and np.array_equal(n1[k, : l1[k]], rn[j, : rl[j]]))
        for j, k in enumerate(pick))
    # E_relaxed on the same sample: in-box out-edges of the nodes settled
    # before the target (distance below the target's), against the box edges
    # the sweep's edge rate counts
    esrc = lat.edge_src()
    xs, ys, zs = (np.asarray(v) for v in lat.coords(np.arange(lat.N)))
    relaxed = boxed = 0
    for k in pick:
        bx = boxes[k]
        inbox = ((xs >= bx[0]) & (xs <= bx[1]) & (ys >= bx[2]) & (ys <= bx[3]) & (zs >= bx[4]) & (zs <= bx[5]))
        g2r = np.where(inbox, np.arange(lat.N), -1).astype(np.int32)
        _, dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(src[k])], dst=int(dst[k]), roi_map=g2r)
        dd = dist[int(dst[k])]
        settled = np.isfinite(dist) & (dist <= dd) & inbox
        e_in = inbox[esrc] & inbox[lat.indices]
        relaxed += int((settled[esrc] & e_in).sum())
        boxed += int(e_in.sum())
    relaxed_frac = relaxed / max(1, boxed)
    return {
        "workload": f"{nsearch} box searches on a 400x400x16 lattice, sides log-uniform per axis "
                    "(x,y 20..400, z 4..16), 3% blocked, shared fp32 costs",
        "mean_roi_nodes": int(vol.mean()),
        "roi_edges_total": roi_edges,
        "searches_per_s_one_per_launch": round(nsearch / t_single, 1),
        "searches_per_s_default_plan": round(nsearch / t_default, 1),
        "searches_per_s_tuned": round(nsearch / t_tuned, 1),
        "box_edges_per_s_tuned": round(roi_edges / t_tuned / 1e9, 3),
        "box_edges_unit": "G directed ROI edges of all searches per second",
        "gteps_tuned": round(relaxed_frac * roi_edges / t_tuned / 1e9, 3),
        "gteps_unit": "G E_relaxed per second: in-box out-edges of the nodes settled before each target, "
                      "as a fraction of the box edges measured by the oracle on the 64-search sample "
                      f"({relaxed_frac:.3f}) and applied to all box edges",
        "speedup_tuned_vs_one_per_launch": round(t_single / t_tuned, 2),
        "sec_tuning": round(t_tune, 2),
        "plan": [{k: v for k, v in b.items()} for b in tune.plan],
        "identical_paths": bool(same and same_single),
        "identical_to_oracle": bool(same_oracle),
        "oracle_sample": "64 of the searches, C heap Dijkstra (fp32) on the same boxes",
    }


def run_ours(args, world, rank, local):
    import torch

    from orthoroute_b200 import _lib
    from orthoroute_b200.build import build_library
    from orthoroute_b200.solver import DeviceGraph

    build_library()
    lib = _lib.load()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lat, w, sources = make_workload(SEED + 7919 * rank, args.nx, args.ny, args.nz, args.sources)
    dg = DeviceGraph.from_lattice(lat, device=dev)
    wt = torch.from_numpy(w).to(dev)
    dist = torch.empty(lat.N, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    # parity before timing: every source's distances bit-exact vs the oracle
    parity = None
    if rank == 0 and not args.no_check:
        parity = parity_all_sources(dg, wt, lat, w, sources, threads=os.cpu_count() or 1,
                                    per_launch=min(args.per_launch, len(sources)))
        if not parity["identical_to_oracle"]:
            raise SystemExit("parity check failed: distances differ from the oracle")

    # algorithmic work per source (from the distances, outside the timed region)
    deg_d = torch.from_numpy(np.diff(lat.indptr).astype(np.int64)).to(dev)
    per_src = []
    for s in sources:
        dg.sssp(wt, int(s), -1, dist_out=dist)
        settled = torch.isfinite(dist)
        per_src.append((int(deg_d[settled].sum().item()), int(settled.sum().item())))
    e_relaxed = sum(e for e, _ in per_src)
    bytes_alg = sum(12 * e + 16 * n for e, n in per_src)

    # The weights stay unchanged through the timed steps: every search
    # declares generation 1 of them, so the whole-lattice weight gather runs
    # once, not once per source (orsp_graph_cost_generation).
    # Headline step (per_launch > 0): orsp_sssp_sources, per_launch sources
    # per launch, each with its own distance row (all rows stay in HBM).
    # The one-source-at-a-time sweep is timed beside it ("single_search").
    per = min(args.per_launch, len(sources)) if args.per_launch > 0 else 0
    dist_all = torch.empty(len(sources), lat.N, dtype=torch.float32, device=dev) if per else None

    def single_step(prof=None):
        for s in sources:
            dg.sssp(wt, int(s), -1, dist_out=dist, cost_generation=1)
            if prof is not None:
                prof()

    def batch_step(prof=None):
        for a in range(0, len(sources), per):
            dg.sssp_sources(wt, sources[a:a + per], dist_all[a:a + per], per_launch=per, cost_generation=1)
            if prof is not None:
                prof()

    kms = ctypes.c_float()
    c8 = (ctypes.c_int64 * 8)()
    acc = {"ms": 0.0, "visits": 0, "n": 0}

    def prof():
        lib.orsp_profile_last(ctypes.byref(kms))
        lib.orsp_profile_counters(c8)
        acc["ms"] += kms.value
        acc["visits"] += int(c8[1])
        acc["n"] += 1

    def timed(step_fn, with_clocks):
        for _ in range(args.warmup):
            step_fn()
        acc.update(ms=0.0, visits=0, n=0)
        lib.orsp_profile_enable(1)
        clocks = clock_sampler(dev) if with_clocks else None
        barrier(world)
        torch.cuda.synchronize(dev)
        if clocks:
            clocks.start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step_fn(prof)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        clk = clocks.stop() if clocks else None
        lib.orsp_profile_enable(0)
        return reduce_max(ev0.elapsed_time(ev1), world), dict(acc), clk

    total_edges = reduce_sum(e_relaxed * args.steps, world)
    ntiles = ((lat.nx + 15) // 16) * ((lat.ny + 15) // 16)
    s_ms, s_acc, s_clk = timed(single_step, with_clocks=not per)
    single = {"ms_per_search": round(s_ms / args.steps / len(sources), 4),
              "gteps": round(total_edges / (s_ms / 1e3) / 1e9, 4),
              "avg_launch_ms": round(s_acc["ms"] / max(1, s_acc["n"]), 4),
              "visits_per_tile": round(s_acc["visits"] / max(1, s_acc["n"]) / ntiles, 2)}
    if per:
        ms_max, b_acc, clk = timed(batch_step, with_clocks=True)
        launches = b_acc["n"]
        kernel_ms = b_acc["ms"]
        srcs_per_launch = len(sources) * args.steps / launches
        visits_per_tile = b_acc["visits"] / (len(sources) * args.steps) / ntiles
    else:
        ms_max, clk = s_ms, s_clk
        launches = s_acc["n"]
        kernel_ms = s_acc["ms"]
        srcs_per_launch = 1
        visits_per_tile = single["visits_per_tile"]
    value = total_edges / (ms_max / 1e3) / 1e9
    # the tile-search kernel of the timed step: many-source launches of up
    # to 12 layers take the warp-specialised schedule (ORSP_LAT_SPEC overrides)
    spec_env = os.environ.get("ORSP_LAT_SPEC")
    spec = (spec_env not in (None, "") and spec_env != "0") if spec_env not in (None, "") else bool(per and lat.nz <= 12)
    timed_kernel = "lattice_spec_kernel" if spec else "lattice_async_kernel"
    avg_kernel_ms = kernel_ms / launches
    bytes_per_launch = bytes_alg / len(sources) * srcs_per_launch
    achieved = bytes_per_launch / (avg_kernel_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # end to end through the public API with host buffers: each step uploads
    # the weights and reads every search's distances back; the read-back of
    # search i (copy stream, two device and two pinned host buffers) overlaps
    # search i + 1
    w_pin = torch.from_numpy(w).pin_memory()
    copy_stream = torch.cuda.Stream(device=dev)
    for _ in range(1):
        wt.copy_(w_pin, non_blocking=True)
    rows = per if per else 1
    d_pin = [torch.empty(rows, lat.N, dtype=torch.float32).pin_memory() for _ in range(2)]
    dbuf = [dist_all, dist_all] if per else [dist.view(1, -1), torch.empty_like(dist).view(1, -1)]
    done = [torch.cuda.Event(), torch.cuda.Event()]
    barrier(world)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps = max(1, min(args.steps, 3))
    k = 0
    for step_i in range(e2e_steps):
        wt.copy_(w_pin, non_blocking=True)
        gen = 1000 + step_i  # new weights every step: gathered once per step
        for a in range(0, len(sources), rows):
            b = k & 1
            if per:  # chunk a of the sources into its own rows of dist_all
                dg.sssp_sources(wt, sources[a:a + rows], dist_all[a:a + rows], per_launch=rows,
                                cost_generation=gen)
                out = dist_all[a:a + rows]
            else:
                stream.wait_event(done[b])  # the buffer's previous read-back has finished
                dg.sssp(wt, int(sources[a]), -1, dist_out=dbuf[b].view(-1), cost_generation=gen)
                out = dbuf[b]
            ready = torch.cuda.Event()
            ready.record(stream)
            copy_stream.wait_event(ready)
            with torch.cuda.stream(copy_stream):
                d_pin[b][: out.shape[0]].copy_(out, non_blocking=True)
                done[b].record(copy_stream)
            k += 1
    stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    e2e_ms = reduce_max(e0.elapsed_time(e1), world)
    e2e_value = reduce_sum(e_relaxed * e2e_steps, world) / (e2e_ms / 1e3) / 1e9

    routing = None
    if not args.no_route:
        with_cpu = rank == 0 and world == 1 and not args.no_cpu
        routing = {"c1": route_c1(dev, with_cpu=with_cpu)}
        if world == 1:
            routing["dropin"] = route_dropin(dev, with_cpu=with_cpu)
            routing["roi_searches"] = roi_searches(dev)
            routing["c3"] = route_c3(dev, with_cpu=with_cpu)
    batch_sweep = sweep_c4(dev) if (world == 1 and not args.no_sweep) else None
    result = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded lattice and weights)",
        "config": workload_config(args, lat, len(sources), world),
        "sources_per_launch": per if per else 1,
        "e2e": {"value": round(e2e_value, 4), "unit": "GTEPS",
                "h2d_bytes_per_step": int(w.nbytes), "d2h_bytes_per_step": int(lat.N * 4 * len(sources))},
        # per launch: fill, seed and the tile search (the weight gather ran
        # before the timed region, once for the unchanged weights)
        "gpu_launches": int(launches * 3),
        "single_search": single,
        "visits_per_tile": round(visits_per_tile, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5),
                     "traffic": int(LAT_DRAM_BYTES_PER_NODE * lat.N * srcs_per_launch),
                     "traffic_source": "ncu dram bytes of a 4-source launch of this lattice, scaled by sources per launch",
                     "kernel": timed_kernel, "peak_kind": peak_kind,
                     "bytes_per_launch": int(bytes_per_launch),
                     "avg_launch_ms": round(avg_kernel_ms, 4)},
        "clocks": clk,
        "parity": parity,
        "routing": routing,
        "batch_sweep": batch_sweep,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        result["cpu_baseline"] = cpu_baseline(lat, w, sources, threads=os.cpu_count() or 1)
    return result


def run_reference(args, world, rank, local):
    """The reference's CPU implementation of the path (the oracle port of
    SimpleDijkstra, C, one source per host thread) on the same workload."""
    if rank != 0:
        return None
    import oracle as O
    from concurrent.futures import ThreadPoolExecutor

    O.build_oracle()
    lat, w, sources = make_workload(SEED, args.nx, args.ny, args.nz, args.sources)
    deg = np.diff(lat.indptr)
    threads = os.cpu_count() or 1

    def one(s):
        _, dist, _, _ = O.dijkstra(lat.indptr, lat.indices, w, [int(s)])
        return int(deg[np.isfinite(dist)].sum())

    sample = list(sources[:threads])
    with ThreadPoolExecutor(max_workers=threads) as ex:
        for _ in range(args.warmup):
            list(ex.map(one, sample[:1]))
        t0 = time.perf_counter()
        edges = 0
        for _ in range(args.steps):
            edges += sum(ex.map(one, sample))
        t = time.perf_counter() - t0
    v = edges / t / 1e9
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 6),
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded lattice and weights)",
        "config": workload_config(args, lat, len(sources), world),
        "cpu_baseline": {"value": round(v, 6), "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"{len(sample)} full searches per step, one per host thread"},
        "e2e": {"value": round(v, 6), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def profile_case(args):
    """A small case of the timed kernel for ncu captures: the bench lattice
    and weights, three orsp_sssp_sources launches of --per-launch new sources
    each (capture the third: -k regex:lattice_async -s 2 -c 1).  Prints one
    line; no timing."""
    import torch

    from orthoroute_b200.build import build_library
    from orthoroute_b200.solver import DeviceGraph

    build_library()
    per = max(1, args.per_launch)
    lat, w, sources = make_workload(SEED, args.nx, args.ny, args.nz, 3 * per)
    dev = torch.device("cuda", 0)
    dg = DeviceGraph.from_lattice(lat, device=dev)
    wt = torch.from_numpy(w).to(dev)
    dist = torch.empty(per, lat.N, dtype=torch.float32, device=dev)
    for k in range(3):
        dg.sssp_sources(wt, sources[k * per:(k + 1) * per], dist, per_launch=per, cost_generation=1)
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_case": f"{args.nx}x{args.ny}x{args.nz}", "launches": 3, "sources_per_launch": per,
                      "settled_last_row": int(torch.isfinite(dist[-1]).sum().item())}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nz", type=int, default=NZ)
    ap.add_argument("--sources", type=int, default=NSRC)
    ap.add_argument("--per-launch", type=int, default=PER_LAUNCH,
                    help="sources per tile-search launch (orsp_sssp_sources); 0: one search per launch")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-check", action="store_true", help="skip the parity check before timing")
    ap.add_argument("--no-route", action="store_true", help="skip the routing measurements")
    ap.add_argument("--no-sweep", action="store_true", help="skip the batched uneven-ROI sweep")
    ap.add_argument("--profile-case", action="store_true",
                    help="run three --per-launch source launches for an ncu capture and exit")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args)
        return
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            res = run_reference(args, world, rank, local)
        else:
            res = run_ours(args, world, rank, local)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
