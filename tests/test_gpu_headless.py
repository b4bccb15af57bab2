"""Headless routing end to end on the GPU: a board written as .ORP, routed by
orthoroute_b200.headless into an .ORS file, against the oracle routing the
same problem on the CPU (same grid, tasks and negotiation schedule) with the
oracle's geometry emission mapped to board coordinates."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from oracle.geometry import emit  # noqa: E402
from oracle.negotiate import route_plain  # noqa: E402
from orthoroute_b200.geometry import _quantize  # noqa: E402
from orthoroute_b200.headless import build_problem, headless_config, run_headless  # noqa: E402
from orthoroute_b200.lattice import board_uniform_pins  # noqa: E402
from orthoroute_b200.orp import orp_to_board_data, read_orp, synthetic_board_data, write_orp  # noqa: E402
from orthoroute_b200.ors import read_ors  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["batched", "sequential"])
def test_headless_orp_to_ors_matches_oracle(tmp_path, mode):
    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    orp = tmp_path / "board.orp"
    ors = tmp_path / "board.ors"
    write_orp(synthetic_board_data(b), orp)
    s = run_headless(str(orp), str(ors), max_iterations=30, mode=mode, log=None)
    geom, meta = read_ors(ors)

    prob = build_problem(orp_to_board_data(read_orp(orp)))
    lat = prob.lattice
    ref = route_plain(lat, prob.src, prob.dst, headless_config(30))
    assert s["converged"] == bool(ref["converged"]) and s["converged"]
    assert meta["statistics"]["converged"] is True

    def xy(node):
        r = int(node) % (lat.nx * lat.ny)
        return (float(_quantize(prob.grid_min_x + (r % lat.nx) * prob.pitch, prob.grid_min_x, prob.pitch)),
                float(_quantize(prob.grid_min_y + (r // lat.nx) * prob.pitch, prob.grid_min_y, prob.pitch)))

    expect_t, expect_v = {}, {}
    for name, (tracks, vias) in zip(prob.names, emit(ref["paths"], lat.nx, lat.ny, lat.nz, prob.layer_dirs)):
        expect_t[name] = [(prob.layer_names[z], xy(a), xy(c)) for a, c, z in tracks]
        # the router's via dicts name the lower layer first
        expect_v[name] = [(xy(n), prob.layer_names[min(z0, z1)], prob.layer_names[max(z0, z1)])
                          for n, z0, z1 in vias]
    got_t = {n: [(t["layer"], (t["start"]["x"], t["start"]["y"]), (t["end"]["x"], t["end"]["y"]))
                 for t in d["tracks"]] for n, d in geom["by_net"].items()}
    got_v = {n: [((v["position"]["x"], v["position"]["y"]), v["from_layer"], v["to_layer"]) for v in d["vias"]]
             for n, d in geom["by_net"].items()}
    for name in prob.names:
        assert got_t.get(name, []) == expect_t[name], name
        assert got_v.get(name, []) == expect_v[name], name
    assert meta["statistics"]["total_tracks"] == sum(len(v) for v in expect_t.values())
    assert meta["statistics"]["total_vias"] == sum(len(v) for v in expect_v.values())
    assert np.isfinite(s["seconds_total"])
