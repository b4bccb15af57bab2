"""The headless board mapping and pad escapes (orthoroute_b200.headless,
orthoroute_b200.escapes) against the reference's own router set-up and
PadEscapePlanner on seeded random boards (CPU only; needs the reference
source tree and is skipped where it is absent).  The escape boards mix
clearance-set footprints, pads of several sizes, pads slightly off their grid
column (kept, with a 45-degree stub tail) and far off it (dropped), and
one-pad obstacle nets, so that column planning, shortening, the clearance
checks and the random entry layers all come into play.  The mapping boards
mix component pads with repeated names, componentless pads with and without
ids, pads on other layers and pads on grid-rounding ties."""
import importlib.util
import json
import logging
import os
import sys
from pathlib import Path

import numpy as np
import pytest

# the reference source tree, named by ORTHOROUTE_REFERENCE (skipped when unset)
REF = Path(os.environ.get("ORTHOROUTE_REFERENCE") or "/nonexistent")
pytestmark = pytest.mark.skipif(not (REF / "orthoroute").exists(), reason="reference source tree not available")
HERE = Path(__file__).resolve().parent


def _golden_module():
    spec = importlib.util.spec_from_file_location("make_golden_orp_ors", HERE / "golden" / "make_golden_orp_ors.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def random_board(seed: int, rows: int = 30) -> dict:
    """rows: the span of footprint origins in grid rows (tall boards put many
    pads, far apart, in the same columns)."""
    rng = np.random.default_rng(seed)
    nz = int(rng.choice([2, 4, 6]))
    names = ["F.Cu"] + [f"In{i}.Cu" for i in range(1, nz - 1)] + ["B.Cu"]
    pads, nets = [], {}

    def pad(net, x, y, w=0.3, h=0.3):
        p = {"component": "", "name": "", "net_name": net, "net_code": 0, "x": round(float(x), 4),
             "y": round(float(y), 4), "width": float(w), "height": float(h), "drill": None, "layers": ["F.Cu"],
             "type": "smd"}
        pads.append(p)
        nets.setdefault(net, {"name": net, "code": 0, "pads": []})["pads"].append(p)

    # two to four footprints: rows x columns of pads at one grid step
    nfp = int(rng.integers(2, 5))
    sites = []
    for f in range(nfp):
        x0 = 20.0 + 0.4 * int(rng.integers(0, 12 if rows > 30 else 30))
        y0 = 20.0 + 0.4 * int(rng.integers(0, rows))
        rows, cols = int(rng.integers(1, 3)), int(rng.integers(3, 9))
        w = float(rng.choice([0.25, 0.3, 0.45]))
        for c in range(cols):
            for r in range(rows):
                sites.append((x0 + 0.4 * c, y0 + 0.4 * r * int(rng.integers(1, 4)), w))
    order = rng.permutation(len(sites))
    for k in range(len(sites) // 2):
        for s in (sites[order[2 * k]], sites[order[2 * k + 1]]):
            pad(f"N{k}", s[0], s[1], s[2], s[2])
    # pads off their grid column: 0.1 step (kept) and 0.3 step (dropped)
    for m in range(3):
        off = 0.04 if m % 2 == 0 else 0.12
        pad(f"OFF{m}", 20.0 + 0.4 * int(rng.integers(0, 30)) + off, 20.0 + 0.4 * int(rng.integers(0, 30)))
        pad(f"OFF{m}", 20.0 + 0.4 * int(rng.integers(0, 30)), 20.0 + 0.4 * int(rng.integers(0, 30)))
    # one-pad obstacle nets in the escape paths
    for m in range(int(rng.integers(3, 8))):
        pad(f"OBS{m}", 20.0 + 12.0 * float(rng.random()), 20.0 + 12.0 * float(rng.random()),
            float(rng.choice([0.3, 0.6])), float(rng.choice([0.3, 0.6])))
    return {"filename": f"random{seed}.kicad_pcb", "x_min": 15.0, "y_min": 15.0, "x_max": 40.0,
            "y_max": 25.0 + 0.4 * rows, "width": 25.0, "height": 10.0 + 0.4 * rows, "layers": nz,
            "layer_names": names, "pads": pads, "nets": nets, "grid_resolution": 0.4}


@pytest.fixture(scope="module")
def reference():
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.dont_write_bytecode = True
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    logging.disable(logging.CRITICAL)
    import orthoroute.algorithms.manhattan.unified_pathfinder as upf
    from orthoroute.domain.models.board import Board, Component, Coordinate, Net, Pad

    return _golden_module(), upf, (Board, Net, Pad, Component, Coordinate)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed,rows", [(11, 30), (12, 30), (13, 30), (14, 30), (15, 30), (16, 30), (17, 160),
                                       (18, 160)])
def test_pad_escapes_equal_reference_on_random_boards(reference, seed, rows):
    from orthoroute_b200.headless import build_problem

    gmod, upf, models = reference
    bd = json.loads(json.dumps(random_board(seed, rows)))
    ref = gmod.reference_portals(bd, upf, models)
    prob = build_problem(bd, portals=True)
    got = [[pid, p.x_idx, p.y_idx, p.pad_layer, p.delta_steps, p.direction, p.pad_x, p.pad_y, p.entry_layer]
           for pid, p in prob.portals.items()]
    assert len(ref["portals"]) > 0
    assert got == ref["portals"]
    assert json.loads(json.dumps(prob.escape_tracks)) == ref["escape_tracks"]
    tasks = {n: [int(s), int(d)] for n, s, d in zip(prob.names, prob.src, prob.dst)}
    assert list(tasks.items()) == list(ref["tasks"].items())
    assert {k: int(v) for k, v in prob.trivial.items()} == ref["trivial"]


def random_component_board(seed: int) -> dict:
    """Named component pads on random layers, repeated pad names within a
    component (the later pad keeps the key), componentless pads with and
    without ids, pads near grid-rounding ties, nets of one to four pads."""
    rng = np.random.default_rng(seed)
    nz = int(rng.choice([2, 3, 4, 8]))
    names = ["F.Cu"] + [f"In{i}.Cu" for i in range(1, nz - 1)] + ["B.Cu"]
    pads, nets, comps = [], {}, []
    for c in range(int(rng.integers(2, 6))):
        comps.append({"reference": f"U{c}", "x": 30.0, "y": 30.0})
    for n in range(int(rng.integers(6, 16))):
        net = f"S{n}"
        for m in range(int(rng.integers(1, 5))):
            kind = rng.integers(0, 4)
            x = 20.0 + 15.0 * float(rng.random())
            y = 20.0 + 15.0 * float(rng.random())
            if kind == 3:  # on a rounding tie of the 0.4 grid
                x = 20.0 + 0.4 * int(rng.integers(0, 30)) + 0.2
            p = {"net_name": net, "net_code": n, "x": round(x, 3), "y": round(y, 3), "width": 0.3, "height": 0.3,
                 "drill": None, "type": "smd",
                 "layers": [names[int(rng.integers(0, nz))]] if rng.random() < 0.5 else ["F.Cu"]}
            if kind == 0:
                p.update(component="", name="")
            elif kind == 1:
                p.update(component="", name="", id=f"P{n}_{m}")
            else:
                p.update(component=f"U{int(rng.integers(0, len(comps)))}", name=str(int(rng.integers(1, 6))))
            pads.append(p)
            nets.setdefault(net, {"name": net, "code": n, "pads": []})["pads"].append(p)
    return {"filename": f"comp{seed}.kicad_pcb", "x_min": 15.0, "y_min": 15.0, "x_max": 40.0, "y_max": 40.0,
            "width": 25.0, "height": 25.0, "layers": nz, "layer_names": names, "pads": pads, "nets": nets,
            "components": comps, "grid_resolution": 0.4}


@pytest.mark.timeout(600)
@pytest.mark.parametrize("seed", [21, 22, 23, 24, 25, 26])
def test_headless_mapping_equals_reference_on_random_boards(reference, seed):
    """Grid, layer directions, pad-to-pad tasks (dict order) and one-node
    routes against the reference router's set-up of the same board."""
    from orthoroute_b200.headless import build_problem

    gmod, upf, models = reference
    bd = json.loads(json.dumps(random_component_board(seed)))
    m = gmod.reference_mapping(bd, upf, models)
    prob = build_problem(bd, pitch=m["pitch"])
    lat = prob.lattice
    assert (lat.nx, lat.ny, lat.nz) == (m["x_steps"], m["y_steps"], m["layers"])
    assert prob.grid_min_x == m["grid_min_x"] and prob.grid_min_y == m["grid_min_y"]
    assert prob.layer_dirs == m["layer_directions"]
    tasks = {n: [int(s), int(d)] for n, s, d in zip(prob.names, prob.src, prob.dst)}
    assert list(tasks.items()) == list(m["tasks"].items())
    assert {k: int(v) for k, v in prob.trivial.items()} == m["trivial"]
