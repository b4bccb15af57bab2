"""The recorded reference run (tests/golden/golden_dropin_tape.npz, made by
tests/golden/make_golden_dropin.py from the unmodified reference router on
the 100x100x4 board with 200 nets) replayed through the CPU oracle: every
accountant update, ROI, search, path -> edge mapping and via step of the
reference's negotiation loop, in the loop's order, must give the
reference's result.  This pins the oracle on the reference's real call
stream; tests/test_gpu_dropin.py replays the same tape through the CUDA
drop-in."""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from oracle.dropin_tape import OracleBackend
from orthoroute_b200.tape import Tape, replay
from orthoroute_b200.lattice import build_lattice

TAPE = Path(__file__).resolve().parent / "golden" / "golden_dropin_tape.npz"


@pytest.fixture(scope="module")
def tape():
    O.build_oracle()
    return Tape.load(TAPE)


def test_tape_is_the_benchmark_board(tape):
    m = tape.meta
    lat = build_lattice(m["nx"], m["ny"], m["nz"])
    assert (lat.N, lat.E) == (m["N"], m["E"])
    kinds = {ev["k"] for ev in tape.events}
    assert {"acct", "roi", "search", "p2e", "via_pen", "via_block"} <= kinds
    assert [t[0] for t in m["trace"]] == list(range(1, m["iterations"] + 1))


@pytest.mark.timeout(900)
def test_oracle_replays_the_reference_tape(tape):
    m = tape.meta
    lat = build_lattice(m["nx"], m["ny"], m["nz"])
    be = OracleBackend(lat.indptr, lat.indices, lat.nx, lat.ny, lat.nz)
    rep = replay(tape, be)
    assert not rep.failures, rep.failures[:5]
    assert rep.searches == sum(1 for ev in tape.events if ev["k"] == "search")
    assert rep.paths_equal_oracle == rep.searches
    # per-iteration overuse of the replayed accounting = the reference's trace
    overs = [ev["out"] for ev in tape.events if ev["k"] == "acct" and ev["m"] == "compute_overuse"]
    assert [tuple(o) for o in overs[-len(m["trace"]):]] == [(s, c) for _, s, c in m["trace"]]
