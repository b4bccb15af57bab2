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


def _expected(prob, paths):
    """Per net: (layer, start, end) of its tracks and (position, lower layer,
    upper layer) of its vias, from the oracle's geometry emission of the
    given paths mapped to board coordinates, escape stubs in front."""
    lat = prob.lattice

    def xy(node):
        r = int(node) % (lat.nx * lat.ny)
        return (float(_quantize(prob.grid_min_x + (r % lat.nx) * prob.pitch, prob.grid_min_x, prob.pitch)),
                float(_quantize(prob.grid_min_y + (r // lat.nx) * prob.pitch, prob.grid_min_y, prob.pitch)))

    expect_t, expect_v = {}, {}
    for t in prob.escape_tracks:
        expect_t.setdefault(t["net"], []).append((t["layer"], (t["x1"], t["y1"]), (t["x2"], t["y2"])))
    for name, (tracks, vias) in zip(prob.names, emit(paths, lat.nx, lat.ny, lat.nz, prob.layer_dirs)):
        expect_t.setdefault(name, []).extend((prob.layer_names[z], xy(a), xy(c)) for a, c, z in tracks)
        # the router's via dicts name the lower layer first
        expect_v[name] = [(xy(n), prob.layer_names[min(z0, z1)], prob.layer_names[max(z0, z1)])
                          for n, z0, z1 in vias]
    return expect_t, expect_v


def _check(prob, ref, s, geom, meta):
    assert s["converged"] == bool(ref["converged"]) and s["converged"]
    assert meta["statistics"]["converged"] is True
    expect_t, expect_v = _expected(prob, ref["paths"])
    got_t = {n: [(t["layer"], (t["start"]["x"], t["start"]["y"]), (t["end"]["x"], t["end"]["y"]))
                 for t in d["tracks"]] for n, d in geom["by_net"].items()}
    got_v = {n: [((v["position"]["x"], v["position"]["y"]), v["from_layer"], v["to_layer"]) for v in d["vias"]]
             for n, d in geom["by_net"].items()}
    for name in set(prob.names) | set(expect_t):
        assert got_t.get(name, []) == expect_t.get(name, []), name
        assert got_v.get(name, []) == expect_v.get(name, []), name
    assert meta["statistics"]["total_tracks"] == sum(len(v) for v in expect_t.values())
    assert meta["statistics"]["total_vias"] == sum(len(v) for v in expect_v.values())
    assert np.isfinite(s["seconds_total"])


@pytest.mark.parametrize("mode", ["batched", "sequential"])
def test_headless_orp_to_ors_matches_oracle(tmp_path, mode):
    """Pad-to-pad routing (no escapes)."""
    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    orp = tmp_path / "board.orp"
    ors = tmp_path / "board.ors"
    write_orp(synthetic_board_data(b), orp)
    s = run_headless(str(orp), str(ors), max_iterations=30, mode=mode, log=None, portals=False)
    geom, meta = read_ors(ors)
    prob = build_problem(orp_to_board_data(read_orp(orp)))
    assert not prob.escape_tracks
    ref = route_plain(prob.lattice, prob.src, prob.dst, headless_config(30))
    _check(prob, ref, s, geom, meta)


@pytest.mark.parametrize("mode", ["batched", "sequential"])
def test_headless_portals_match_oracle(tmp_path, mode):
    """The default portal flow: pads escape to portals (stubs on F.Cu), the
    searches run between the portals' F.Cu nodes, and the .ORS holds the
    stubs in front of each net's routed tracks."""
    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    orp = tmp_path / "board.orp"
    ors = tmp_path / "board.ors"
    write_orp(synthetic_board_data(b), orp)
    s = run_headless(str(orp), str(ors), max_iterations=30, mode=mode, log=None)
    geom, meta = read_ors(ors)
    prob = build_problem(orp_to_board_data(read_orp(orp)), portals=True)
    assert s["portals"] == len(prob.portals) > 0 and s["escape_tracks"] == len(prob.escape_tracks)
    plane = prob.lattice.nx * prob.lattice.ny
    assert np.all(prob.search_src < plane) and np.all(prob.search_dst < plane)  # F.Cu seeds
    ref = route_plain(prob.lattice, prob.search_src, prob.search_dst, headless_config(30))
    _check(prob, ref, s, geom, meta)


@pytest.mark.parametrize("mode", ["batched", "sequential"])
@pytest.mark.parametrize("vias", ["full", "adjacent"])
def test_headless_via_sets_match_oracle(tmp_path, mode, vias):
    """The portal flow on both via sets: the reference's (F.Cu to every
    routing layer, every pair of routing layers; the default, searched as a
    column-via lattice, batched on the tile sweeps) and adjacent-layer vias
    (the device routing loop in sequential mode); every net's stubs, tracks
    and vias equal the oracle loop's on the same lattice."""
    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    orp = tmp_path / "board.orp"
    ors = tmp_path / "board.ors"
    write_orp(synthetic_board_data(b), orp)
    s = run_headless(str(orp), str(ors), max_iterations=30, mode=mode, log=None, vias=vias)
    geom, meta = read_ors(ors)
    prob = build_problem(orp_to_board_data(read_orp(orp)), portals=True, vias=vias)
    assert s["lattice_vias"] == vias and (vias == "adjacent" or s["forced_overuse"] == 0)
    ref = route_plain(prob.lattice, prob.search_src, prob.search_dst, headless_config(30))
    _check(prob, ref, s, geom, meta)


@pytest.mark.parametrize("vias", ["full", "adjacent"])
def test_headless_snapshot_groups_match_oracle(tmp_path, vias):
    """`--groups`: the portal flow routed in snapshot groups of 8 nets with
    3 repair rounds (orsp_route_nets_snapshot, on the column-via lattice of
    the reference's via set or on adjacent vias); every net's stubs, tracks
    and vias equal the oracle loop's of the same schedule."""
    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    orp = tmp_path / "board.orp"
    ors = tmp_path / "board.ors"
    write_orp(synthetic_board_data(b), orp)
    s = run_headless(str(orp), str(ors), max_iterations=30, mode="batched", log=None, vias=vias, groups=8)
    geom, meta = read_ors(ors)
    prob = build_problem(orp_to_board_data(read_orp(orp)), portals=True, vias=vias)
    assert s["snapshot_groups"] == 8
    ref = route_plain(prob.lattice, prob.search_src, prob.search_dst, headless_config(30, groups=8))
    _check(prob, ref, s, geom, meta)
