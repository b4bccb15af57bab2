"""The .ORP / .ORS formats and the headless board mapping against golden files
written by the reference's own exporter, importer and router set-up
(tests/golden/make_golden_orp_ors.py).  No GPU needed."""
import gzip
import json
from pathlib import Path

import numpy as np
import pytest

from orthoroute_b200.headless import build_problem, merge_escapes
from orthoroute_b200.lattice import board_uniform_pins
from orthoroute_b200.orp import (board_data_to_orp, orp_to_board_data, read_orp, synthetic_board_data,
                                 write_orp)
from orthoroute_b200.ors import ors_to_geometry_payload, read_ors, solution_to_ors, write_ors

GOLDEN = Path(__file__).resolve().parent / "golden"


def _json(o):
    return json.loads(json.dumps(o))


def _gz_json(path):
    with gzip.open(path, "rt", encoding="utf-8") as f:
        return json.load(f)


@pytest.fixture(scope="module")
def gorp():
    return json.loads((GOLDEN / "golden_orp.json").read_text())


@pytest.fixture(scope="module")
def gors():
    return json.loads((GOLDEN / "golden_ors.json").read_text())


@pytest.mark.parametrize("suffix", ["", "_2l", "_fp"])
def test_read_and_convert_reference_orp(gorp, suffix):
    """A file the reference wrote reads back as the reference reads it, and
    converts to the reference's board_data."""
    path = GOLDEN / f"golden_board{suffix}.orp"
    doc = read_orp(path)
    assert doc == _gz_json(path)
    assert _json(orp_to_board_data(doc)) == gorp["converted" + suffix]


@pytest.mark.parametrize("suffix", ["", "_2l", "_fp"])
def test_write_orp_matches_reference(gorp, suffix):
    """board_data -> ORP document: the reference's, field for field (the
    export time aside)."""
    name = f"golden_board{suffix}.orp"
    ref = _gz_json(GOLDEN / name)
    ts = ref["metadata"]["export_timestamp"]
    ours = board_data_to_orp(gorp["board_data" + suffix], filename=name, timestamp=ts)
    assert _json(ours) == ref


@pytest.mark.parametrize("suffix", ["", "_2l", "_fp"])
def test_headless_mapping_matches_reference(gorp, suffix):
    """Grid, layer directions, pad-to-pad tasks (dict order) and one-node
    routes of the reference's router set-up on the same board: a 6-layer
    board, and a 2-layer board with a repeated pad key (the later pad wins,
    as in the reference)."""
    m = gorp["mapping" + suffix]
    prob = build_problem(gorp["converted" + suffix], pitch=m["pitch"])
    lat = prob.lattice
    assert (lat.nx, lat.ny, lat.nz) == (m["x_steps"], m["y_steps"], m["layers"])
    assert prob.grid_min_x == m["grid_min_x"] and prob.grid_min_y == m["grid_min_y"]
    assert prob.layer_dirs == m["layer_directions"]
    tasks = {n: [int(s), int(d)] for n, s, d in zip(prob.names, prob.src, prob.dst)}
    assert list(tasks.items()) == list(m["tasks"].items())
    assert {k: int(v) for k, v in prob.trivial.items()} == m["trivial"]


@pytest.mark.parametrize("suffix", ["", "_2l", "_fp"])
def test_pad_escapes_match_reference(gorp, suffix):
    """Pad escapes and portals (orthoroute_b200.escapes) against the
    reference's PadEscapePlanner in its default headless set-up: the same
    portals in the same order (cell, length, direction, entry layer), the same
    escape stubs, and the same portal-to-portal tasks."""
    g = gorp["portals" + suffix]
    prob = build_problem(gorp["converted" + suffix], portals=True)
    got = [[pid, p.x_idx, p.y_idx, p.pad_layer, p.delta_steps, p.direction, p.pad_x, p.pad_y, p.entry_layer]
           for pid, p in prob.portals.items()]
    assert got == g["portals"]
    assert _json(prob.escape_tracks) == g["escape_tracks"]
    tasks = {n: [int(s), int(d)] for n, s, d in zip(prob.names, prob.src, prob.dst)}
    assert list(tasks.items()) == list(g["tasks"].items())
    assert {k: int(v) for k, v in prob.trivial.items()} == g["trivial"]
    # the searches start and end on the portals' F.Cu nodes (the reference's only seeds)
    plane = prob.lattice.nx * prob.lattice.ny
    nx = prob.lattice.nx
    for name, s0, d0, s, d in zip(prob.names, prob.search_src, prob.search_dst, prob.src, prob.dst):
        k1, k2 = prob.net_pads[name]
        if k1 in prob.portals and k2 in prob.portals:
            a, b = prob.portals[k1], prob.portals[k2]
            if (a.x_idx, a.y_idx) != (b.x_idx, b.y_idx):
                assert (s0, d0) == (a.y_idx * nx + a.x_idx, b.y_idx * nx + b.x_idx)
                assert s0 == s % plane and d0 == d % plane
                continue
        assert (s0, d0) == (s, d)


def test_portal_collisions_counted():
    """Grid points where portals of different nets meet: none on the golden
    boards, and a planted one (a third net's portal moved onto another's)
    counts once."""
    import copy
    import json as _j

    from orthoroute_b200.headless import portal_collisions

    g = _j.loads((GOLDEN / "golden_orp.json").read_text())
    for sfx in ("", "_2l", "_fp"):
        prob = build_problem(g["converted" + sfx], portals=True)
        assert portal_collisions(prob) == 0
    prob = build_problem(g["converted_fp"], portals=True)
    keys = list(prob.portals)
    pad_net = {k: n for n, ks in prob.net_pads.items() for k in ks}
    a = keys[0]
    b = next(k for k in keys if pad_net.get(k) != pad_net.get(a))
    prob.portals[b] = copy.copy(prob.portals[b])
    prob.portals[b].x_idx, prob.portals[b].y_idx = prob.portals[a].x_idx, prob.portals[a].y_idx
    assert portal_collisions(prob) == 1


def test_forced_overuse_bound():
    """F.Cu search endpoints shared in the same direction force overused via
    edges on boards of more than two layers; endpoints shared in opposite
    directions do not, and 2-layer boards have planar F.Cu edges."""
    from orthoroute_b200.headless import forced_overuse

    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    prob = build_problem(orp_to_board_data(board_data_to_orp(synthetic_board_data(b))), portals=True,
                         vias="adjacent")
    assert int(max(prob.search_src.max(), prob.search_dst.max())) < prob.lattice.nx * prob.lattice.ny  # F.Cu
    assert forced_overuse(prob) == 0
    s0, d0 = int(prob.search_src[0]), int(prob.search_dst[0])
    prob.search_dst[1] = s0  # opposite directions: still routable
    assert forced_overuse(prob) == 0
    prob.search_src[2] = s0  # two searches leave s0
    prob.search_dst[3] = d0  # two searches enter d0
    assert forced_overuse(prob) == 2
    b2 = board_uniform_pins(30, 24, 2, 12, seed=3)
    p2 = build_problem(synthetic_board_data(b2), portals=True, vias="adjacent")
    p2.search_src[1] = p2.search_src[0]
    assert forced_overuse(p2) == 0


def test_one_layer_board_routes_pad_to_pad(gorp):
    """A one-layer board has no routing layer for portals: its tasks stay
    pad to pad and every node is inside the lattice."""
    bd = dict(gorp["converted"], layers=1, layer_names=["F.Cu"])
    prob = build_problem(bd, portals=True)
    ref = build_problem(bd)
    assert not prob.portals and not prob.escape_tracks
    assert np.array_equal(prob.src, ref.src) and np.array_equal(prob.search_dst, ref.dst)
    assert prob.lattice.nz == 1 and int(max(prob.src.max(), prob.dst.max())) < prob.lattice.N


def test_merge_escapes_dedupe():
    """Escape stubs go in front; a routed track equal to a stub up to
    0.001 mm is dropped, and so is a repeated via."""
    esc = [{"net": "A", "layer": "F.Cu", "x1": 1.0, "y1": 2.0, "x2": 1.0, "y2": 3.2000004, "width": 0.24}]
    tr = [{"net": "A", "layer": "F.Cu", "x1": 1.0, "y1": 2.0, "x2": 1.0, "y2": 3.2, "width": 0.24},
          {"net": "B", "layer": "F.Cu", "x1": 1.0, "y1": 2.0, "x2": 1.0, "y2": 3.2, "width": 0.24}]
    via = {"net": "A", "x": 1.0, "y": 3.2, "from_layer": "F.Cu", "to_layer": "In1.Cu", "diameter": 0.25,
           "drill": 0.15}
    t, v = merge_escapes(esc, tr, [via, dict(via)])
    assert t == [esc[0], tr[1]] and v == [via]
    assert merge_escapes([], tr, [via, dict(via)]) == (tr, [via, via])


def test_ors_matches_reference(gors, tmp_path):
    """Solution -> ORS document, read back, and back to the router's payload
    form: the reference's results on mixed track / via / metric key styles."""
    inp = gors["inputs"]

    class Payload:
        tracks = inp["tracks"]
        vias = inp["vias"]

    ref = _gz_json(GOLDEN / "golden_solution.ors")
    ts = ref["metadata"]["export_timestamp"]
    ours = solution_to_ors(Payload, inp["metrics"], inp["metadata"], timestamp=ts)
    assert _json(ours) == ref
    geom, meta = read_ors(GOLDEN / "golden_solution.ors")
    assert _json([geom, meta]) == [gors["imported"]["geometry"], gors["imported"]["metadata"]]
    back = ors_to_geometry_payload(geom)
    assert _json([back.tracks, back.vias]) == [gors["payload"]["tracks"], gors["payload"]["vias"]]
    # our own file reads back the same way
    out = tmp_path / "s.ors"
    doc = write_ors(Payload, inp["metrics"], inp["metadata"], out)
    g2, m2 = read_ors(out)
    assert _json(g2) == _json(doc["geometry"]) and _json(m2["statistics"]) == ref["statistics"]


def test_format_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        read_orp(tmp_path / "missing.orp")
    with pytest.raises(FileNotFoundError):
        read_ors(tmp_path / "missing.ors")
    for name, reader in (("a.orp", read_orp), ("a.ors", read_ors)):
        p = tmp_path / name
        p.write_text(json.dumps({"metadata": {}}))
        with pytest.raises(ValueError, match="Missing format_version"):
            reader(p)
        p.write_text(json.dumps({"format_version": "2.0"}))
        with pytest.raises(ValueError, match="Unsupported"):
            reader(p)
        with gzip.open(p, "wt") as f:
            json.dump({"format_version": "1.0", "metadata": {}}, f)
        with pytest.raises(ValueError, match="Missing required sections"):
            reader(p)
    with pytest.raises(ValueError, match="Geometry cannot be None"):
        solution_to_ors(None, [], {})


def test_synthetic_board_round_trip(tmp_path):
    """A benchmark board exported as .ORP maps back onto its own grid cells:
    every pin keeps its (x, y, layer) up to the routing area's offset."""
    b = board_uniform_pins(30, 24, 4, 12, seed=3)
    path = tmp_path / "b.orp"
    write_orp(synthetic_board_data(b), path)
    prob = build_problem(orp_to_board_data(read_orp(path)))
    assert prob.names == b.names
    ox = round((10.0 - prob.grid_min_x) / 0.4)
    oy = round((10.0 - prob.grid_min_y) / 0.4)
    for a, c in ((b.src, prob.src), (b.dst, prob.dst)):
        x, y, z = b.lattice.coords(a)
        px, py, pz = prob.lattice.coords(c)
        assert np.array_equal(px, x + ox) and np.array_equal(py, y + oy) and np.array_equal(pz, z)


def test_full_via_lattice_problem():
    """vias='full' builds the reference's via set (F.Cu to every routing layer
    and every pair of routing layers), which the device recognises as a
    column-via lattice; the same tasks as the adjacent-via lattice, and no
    forced overuse at shared F.Cu endpoints (one via per layer pair)."""
    from orthoroute_b200.headless import forced_overuse

    b = board_uniform_pins(40, 32, 6, 30, seed=5)
    bd = orp_to_board_data(board_data_to_orp(synthetic_board_data(b)))
    pa = build_problem(bd, portals=True, vias="adjacent")
    pf = build_problem(bd, portals=True)
    assert pf.vias == "full" and pa.vias == "adjacent"
    assert np.array_equal(pa.search_src, pf.search_src) and np.array_equal(pa.search_dst, pf.search_dst)
    lat = pf.lattice
    plane = lat.nx * lat.ny
    u = np.repeat(np.arange(lat.N), np.diff(lat.indptr))
    v = lat.indices.astype(np.int64)
    via = (u // plane) != (v // plane)
    pairs = {(int(a), int(c)) for a, c in zip(u[via] // plane, v[via] // plane)}
    routing = range(1, lat.nz - 1)
    want = {(a, c) for a in routing for c in routing if a != c} | {(0, c) for c in routing} | {(c, 0) for c in routing}
    assert pairs == want
    pf.search_src[2] = pf.search_src[0]
    assert forced_overuse(pf) == 0
