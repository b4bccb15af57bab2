"""Records the tape of the unmodified reference router routing the
100x100x4 board (200 two-pin nets, pins uniform on the top layer, seed 1):
every call the negotiation loop makes into the hot path during the first
iterations, with inputs, outputs (arrays as digests) and the reference's
time per call (oracle/dropin_tape.py).  tests/test_dropin_tape.py replays it
through the CPU oracle, and tests/test_gpu_dropin.py through the CUDA
drop-in; bench.py times the replay.

    python tests/golden/make_golden_dropin.py [--ref <OrthoRoute tree>] [--iters 3]
                                              (default --ref: $ORTHOROUTE_REFERENCE)
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

import oracle as O  # noqa: E402
from oracle.dropin_tape import TapeRecorder  # noqa: E402
from oracle.ref_harness import run_reference  # noqa: E402
from orthoroute_b200.lattice import board_uniform_pins  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ORTHOROUTE_REFERENCE"),
                    required=not os.environ.get("ORTHOROUTE_REFERENCE"),
                    help="OrthoRoute source tree (default: $ORTHOROUTE_REFERENCE)")
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--out", default=str(REPO / "tests" / "golden" / "golden_dropin_tape.npz"))
    args = ap.parse_args()
    O.build_oracle()
    nx, ny, nz, nets, seed = 100, 100, 4, 200, 1
    b = board_uniform_pins(nx, ny, nz, nets, seed=seed)
    lat = b.lattice
    holder = {}

    def on_init(router):
        holder["rec"] = TapeRecorder(router, lat.indptr, lat.indices, oracle=O)

    def on_iteration(it, over_sum, over_cnt):
        holder["rec"].iteration_done(it, over_sum, over_cnt)

    t0 = time.perf_counter()
    res = run_reference(lat, b.src, b.dst, ref=args.ref, max_iterations=args.iters, on_init=on_init,
                        on_iteration=on_iteration)
    rec = holder["rec"]
    tape = rec.tape
    tape.meta = {"board": f"{nx}x{ny}x{nz} lattice, {nets} two-pin nets, pins uniform on the top layer",
                 "nx": nx, "ny": ny, "nz": nz, "N": lat.N, "E": lat.E, "nets": nets, "seed": seed,
                 "iterations": args.iters, "trace": res["trace"], "reference_route_seconds": res["seconds"],
                 "pres_fac_init": 0.5, "pres_fac_mult": 1.5, "hist_gain": 1.0,
                 "recorded_in_seconds": time.perf_counter() - t0,
                 "host": "reference timed single-threaded in the recording container"}
    tape.save(args.out)
    kinds = {}
    for ev in tape.events:
        kinds[ev["k"]] = kinds.get(ev["k"], 0) + 1
    differ = sum(1 for ev in tape.events if ev["k"] == "search" and "oracle" in ev)
    print(f"wrote {args.out}: {len(tape.events)} events {kinds}, {len(tape.blobs)} blobs, "
          f"{differ} searches where the reference's float64 path differs from the fp32 oracle's; "
          f"trace {res['trace']}")


if __name__ == "__main__":
    main()
