"""Training data, training and evaluation of the history warm start.

    python -m orthoroute_b200.warm_train [--boards 500] [--heldout 50] [--size 200] [--epochs 30]
                                         [--scale-size 600] [--scales 4,16,64] [--rudy-scales 1,4,16]
                                         [--group-nets 32] [--group-repair 3]
                                         [--out orthoroute_b200/data/warm_history.npz]

Boards: seeded connector-footprint boards (2x50-pin footprints, one net per
pin) of size x size cells and 18 layers, with nets at the density of the
600x600x18 backplane (8 000 nets on 360 000 cells); seeds from 2000, so the
benchmark board (seed 3) is never seen.  Each board is routed to zero
overuse by PathFinder with per-net live costs from zero initial history, in
snapshot groups of --group-nets nets with --group-repair repair rounds (the
schedule the prediction later steers; --group-nets 0: one launch per round
of disjoint boxes); its final history field, log1p per node and kind,
averaged over 5x5 cells in x/y, is the training target.  Training takes random 200x200 windows (the net is
fully convolutional).  The history scale used at routing time is chosen on
the held-out boards: the one that converges on most boards with the fewest
iterations (ties: least time).  The defaults reproduce the weights shipped
in orthoroute_b200/data/warm_history.npz (summary in warm_history.json).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path
from typing import List, Optional

import numpy as np
import torch

from .lattice import board_footprints
from .negotiate import NegotiationConfig, PathFinder
from .warm import (WarmNet, board_features, board_features_device, history_from_prediction, node_targets,
                   rudy_prediction)

DENSITY = 8000 / (600 * 600)
DEFAULT_OUT = Path(__file__).resolve().parent / "data" / "warm_history.npz"


# snapshot groups of the routing schedule (0: one launch per round of
# disjoint boxes), set from --group-nets / --group-repair
SCHEDULE = {"group_nets": 0, "group_repair": 0}


def route_config(max_iterations: int = 60) -> NegotiationConfig:
    """The routing schedule of the backplane benchmark."""
    return NegotiationConfig(max_iterations=max_iterations, cost_update="net", reroute="offenders", roi_margin=10,
                             full_graph_retry=False, net_order="disjoint", stall_grow=10, stall_iterations=2,
                             group_nets=SCHEDULE["group_nets"], group_repair=SCHEDULE["group_repair"])


def make_board(size: int, nz: int, seed: int):
    nets = max(8, int(round(DENSITY * size * size)))
    return board_footprints(size, size, nz, nets, None, seed=seed)


def make_sample(size: int, nz: int, seed: int, device=None, blur: int = 2, on_device: bool = False) -> dict:
    """Routes one board with zero history; returns features, targets (the
    final history, blurred over 2 blur + 1 cells in x/y) and stats.  With
    on_device, the features are the padded bf16 device tensor the network
    reads (board_features_device: the same values as board_features after
    the bf16 conversion) and size must be a multiple of 8."""
    b = make_board(size, nz, seed)
    pf = PathFinder(b.lattice, config=route_config(), device=device)
    r = pf.route(b.src, b.dst, mode="batched")
    hist = pf.acc.history.cpu().numpy()
    x = board_features_device(b.lattice, b.src, b.dst, device=pf.device) if on_device else \
        board_features(b.lattice, b.src, b.dst)
    return {"x": x, "t": node_targets(b.lattice, hist, blur),
            "iterations": len(r.iterations), "converged": r.converged, "seconds": r.seconds, "seed": seed}


def _x_device(x) -> torch.Tensor:
    return x if isinstance(x, torch.Tensor) else torch.from_numpy(x).cuda().to(torch.bfloat16)


def _crop(a: torch.Tensor, y0: int, x0: int, c: int) -> torch.Tensor:
    return a[:, y0:y0 + c, x0:x0 + c].contiguous()


def _weights(t: torch.Tensor, boost: float) -> Optional[torch.Tensor]:
    """Per-voxel loss weight: 1, or 1 + boost where the target history is
    non-zero (the field is sparse; most cells never see congestion)."""
    if boost <= 0:
        return None
    return (1.0 + boost * (t.sum(-1) > 1e-3).float()).contiguous()


def train(net: WarmNet, data: List[dict], epochs: int, lr: float = 2e-3, seed: int = 0, log=None,
          crop: int = 0, steps_per_epoch: int = 0, boost: float = 0.0) -> List[float]:
    """Adam with a cosine schedule.  crop > 0: each step takes a random
    crop x crop window (a multiple of 8) of a random board; otherwise one
    step per whole board."""
    rng = np.random.default_rng(seed)
    xs = [_x_device(d["x"]) for d in data]
    ts = [torch.from_numpy(np.ascontiguousarray(d["t"])).cuda() for d in data]
    hist = []
    n_steps = steps_per_epoch if crop else len(data)
    for ep in range(epochs):
        lr_e = lr * 0.5 * (1 + np.cos(np.pi * ep / max(1, epochs)))
        tot = 0.0
        order = rng.permutation(len(data)) if not crop else rng.integers(0, len(data), n_steps)
        for i in order:
            x, t = xs[i], ts[i]
            if crop:
                H, W = x.shape[1], x.shape[2]
                y0 = int(rng.integers(0, H - crop + 1))
                x0 = int(rng.integers(0, W - crop + 1))
                x, t = _crop(x, y0, x0, crop), _crop(t, y0, x0, crop)
            out, act = net.forward(x, keep=True)
            loss, dout = net.loss_grad(out, t, _weights(t, boost))
            net.backward(act, dout)
            net.step(lr=float(lr_e), wd=1e-5)
            tot += float(loss)
        hist.append(tot / max(1, len(order)))
        if log:
            log(f"epoch {ep + 1}/{epochs} loss {hist[-1]:.5f}")
    return hist


def eval_loss(net: WarmNet, data: List[dict]) -> float:
    tot = 0.0
    for d in data:
        out = net.forward(_x_device(d["x"]))
        loss, _ = net.loss_grad(out, torch.from_numpy(np.ascontiguousarray(d["t"])).cuda())
        tot += float(loss)
    return tot / max(1, len(data))


def warm_route(net, board, scale: float, mode: str = "batched", device=None, max_iterations: int = 60):
    """Routes `board` from a predicted history; returns (RouteResult, seconds
    spent on features + prediction + mapping).  `net` is a WarmNet or the
    string "rudy" (the non-learned prior, warm.rudy_prediction)."""
    t0 = time.perf_counter()
    if isinstance(net, str):
        pred = rudy_prediction(board.lattice, board.src, board.dst)
    else:
        pred = net.predict(board_features(board.lattice, board.src, board.dst, net.features))
    h0 = history_from_prediction(board.lattice, pred, scale)
    torch.cuda.synchronize()
    t_pred = time.perf_counter() - t0
    pf = PathFinder(board.lattice, config=route_config(max_iterations), device=device)
    r = pf.route(board.src, board.dst, mode=mode, history_init=h0)
    return r, t_pred


def choose_scale(net, size: int, nz: int, seeds: List[int], scales=(0.25, 0.5, 1.0)) -> dict:
    """The history scale (for a WarmNet or "rudy") that converges on most
    boards with the fewest iterations (ties: least time)."""
    boards = [make_board(size, nz, sd) for sd in seeds]
    res = {}
    for s in scales:
        its, secs, conv = 0, 0.0, 0
        for b in boards:
            r, tp = warm_route(net, b, s)
            its += len(r.iterations)
            secs += r.seconds + tp
            conv += int(r.converged)
        res[s] = {"iterations": its, "seconds": secs, "converged": conv}
    best = min(scales, key=lambda s: (-res[s]["converged"], res[s]["iterations"], res[s]["seconds"]))
    return {"scale": best, "table": res}


def main(argv: Optional[List[str]] = None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--boards", type=int, default=500)
    ap.add_argument("--heldout", type=int, default=50)
    ap.add_argument("--size", type=int, default=200)
    ap.add_argument("--nz", type=int, default=18)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--seed", type=int, default=2000)
    ap.add_argument("--crop", type=int, default=200, help="train on random crop x crop windows (multiple of 8)")
    ap.add_argument("--steps", type=int, default=100, help="steps per epoch when cropping")
    ap.add_argument("--boost", type=float, default=0.0, help="extra loss weight on cells with history")
    ap.add_argument("--blur", type=int, default=2, help="target averaged over (2 blur + 1)^2 cells in x/y")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--scale-boards", type=int, default=2, help="held-out boards used to choose the scale")
    ap.add_argument("--scale-size", type=int, default=600, help="size of those boards (0: --size)")
    ap.add_argument("--scales", default="4,16,64")
    ap.add_argument("--rudy-scales", default="1,4,16", help="scales tried for the RUDY prior (empty: no ablation)")
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    ap.add_argument("--summary", default=None)
    ap.add_argument("--group-nets", type=int, default=32,
                    help="route targets and held-out boards in snapshot groups of this many nets (0: disjoint rounds)")
    ap.add_argument("--group-repair", type=int, default=3, help="repair rounds of the snapshot groups")
    ap.add_argument("--features-on-host", action="store_true",
                    help="keep the boards' features on the host as float32 (default: on the GPU as bf16, size a "
                         "multiple of 8)")
    args = ap.parse_args(argv)
    SCHEDULE["group_nets"] = args.group_nets
    SCHEDULE["group_repair"] = args.group_repair if args.group_nets > 0 else 0
    log = lambda m: print(m, flush=True)  # noqa: E731
    t0 = time.perf_counter()
    seeds = [args.seed + i for i in range(args.boards + args.heldout)]
    data = []
    for i, sd in enumerate(seeds):
        data.append(make_sample(args.size, args.nz, sd, blur=args.blur,
                                on_device=not args.features_on_host and args.size % 8 == 0))
        log(f"routed {i + 1}/{len(seeds)} boards ({data[-1]['iterations']} iterations, "
            f"{data[-1]['seconds']:.1f} s)")
    t_data = time.perf_counter() - t0
    train_set, held = data[: args.boards], data[args.boards:]
    net = WarmNet(C=32, seed=args.seed)
    t1 = time.perf_counter()
    losses = train(net, train_set, args.epochs, lr=args.lr, log=log, crop=args.crop, steps_per_epoch=args.steps,
                   boost=args.boost)
    t_train = time.perf_counter() - t1
    held_loss = eval_loss(net, held)
    zero = WarmNet(C=32, seed=args.seed)
    for k in zero.w:
        zero.w[k].zero_()
    base_loss = eval_loss(zero, held)  # predicting zero history everywhere
    scales = tuple(float(v) for v in args.scales.split(","))
    ssize = args.scale_size or args.size
    sseeds = seeds[args.boards:][: args.scale_boards]
    sc = choose_scale(net, ssize, args.nz, sseeds, scales)
    if ssize == args.size:
        plain_its = sum(d["iterations"] for d in held[: args.scale_boards])
        plain_secs = sum(d["seconds"] for d in held[: args.scale_boards])
    else:  # the scale boards are of another size: route them plainly here
        plain = [make_sample(ssize, args.nz, sd, blur=args.blur) for sd in sseeds]
        plain_its = sum(d["iterations"] for d in plain)
        plain_secs = sum(d["seconds"] for d in plain)
    rudy = None
    if args.rudy_scales:
        rudy = choose_scale("rudy", ssize, args.nz, sseeds, tuple(float(v) for v in args.rudy_scales.split(",")))
    st = net.state()
    st["scale"] = np.float32(sc["scale"])
    st["features"] = np.int32(net.features)
    if rudy is not None:
        st["rudy_scale"] = np.float32(rudy["scale"])
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(args.out, **{k: (v.astype(np.float16) if k.startswith("w_") else v) for k, v in st.items()})
    summary = {"boards": args.boards, "heldout": args.heldout, "size": args.size, "nz": args.nz,
               "epochs": args.epochs, "train_loss": losses, "heldout_loss": held_loss,
               "heldout_loss_zero_prediction": base_loss, "scale": sc["scale"],
               "scale_table": {str(k): v for k, v in sc["table"].items()},
               "scale_boards": {"size": ssize, "seeds": sseeds},
               "rudy_scale": None if rudy is None else rudy["scale"],
               "rudy_scale_table": None if rudy is None else {str(k): v for k, v in rudy["table"].items()},
               "heldout_plain_iterations": plain_its, "heldout_plain_seconds": plain_secs,
               "crop": args.crop, "steps": args.steps, "boost": args.boost, "blur": args.blur, "lr": args.lr,
               "sec_data": round(t_data, 1), "sec_train": round(t_train, 1),
               "group_nets": SCHEDULE["group_nets"], "group_repair": SCHEDULE["group_repair"],
               "plain_iterations_mean": float(np.mean([d["iterations"] for d in data]))}
    log(json.dumps(summary))
    if args.summary:
        Path(args.summary).write_text(json.dumps(summary, indent=1))
    return summary


if __name__ == "__main__":
    main()
