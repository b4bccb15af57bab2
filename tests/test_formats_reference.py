""".ORP and .ORS documents (orthoroute_b200.orp / .ors) against the
reference's own exporters and importers on seeded random inputs (CPU only;
needs the reference source tree and is skipped where it is absent).  Boards
omit optional keys at random (names, sizes, layers, drill, bounds, DRC
values) and solutions mix every track / via / metric key style the
reference's writer accepts."""
import gzip
import json
import logging
import os
import sys
from pathlib import Path

import numpy as np
import pytest

# the reference source tree, named by ORTHOROUTE_REFERENCE (skipped when unset)
REF = Path(os.environ.get("ORTHOROUTE_REFERENCE") or "/nonexistent")
pytestmark = [pytest.mark.skipif(not (REF / "orthoroute").exists(), reason="reference source tree not available"),
              pytest.mark.filterwarnings("ignore::DeprecationWarning")]


@pytest.fixture(scope="module")
def ref_io():
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.dont_write_bytecode = True
    if str(REF) not in sys.path:
        sys.path.insert(0, str(REF))
    logging.disable(logging.CRITICAL)
    from orthoroute.infrastructure.serialization import orp_exporter, ors_exporter

    return orp_exporter, ors_exporter


def _json(o):
    return json.loads(json.dumps(o))


def _gz(path):
    with gzip.open(path, "rt", encoding="utf-8") as f:
        return json.load(f)


def random_board_data(seed: int) -> dict:
    rng = np.random.default_rng(seed)
    nz = int(rng.choice([2, 4, 6]))
    names = ["F.Cu"] + [f"In{i}.Cu" for i in range(1, nz - 1)] + ["B.Cu"]
    pads, nets = [], {}
    for n in range(int(rng.integers(3, 10))):
        net = f"NET{n}"
        for m in range(int(rng.integers(1, 4))):
            p = {"net_name": net, "x": round(float(10 + 30 * rng.random()), 4),
                 "y": round(float(10 + 30 * rng.random()), 4)}
            if rng.random() < 0.8:
                p["component"] = "" if rng.random() < 0.3 else f"R{int(rng.integers(1, 5))}"
            if rng.random() < 0.8:
                p["name"] = str(int(rng.integers(1, 9)))
            if rng.random() < 0.8:
                p["width"] = float(rng.choice([0.2, 0.3, 0.5]))
                p["height"] = float(rng.choice([0.2, 0.3, 0.5]))
            r = rng.random()
            if r < 0.2:
                p["layers"] = list(names)
                p["drill"] = float(rng.choice([0.3, 0.8]))
            elif r < 0.4:
                p["layers"] = ["B.Cu"]
            elif r < 0.5:
                p["layers"] = []
            elif r < 0.8:
                p["layers"] = ["F.Cu"]
            if "drill" not in p and rng.random() < 0.3:
                p["drill"] = None if rng.random() < 0.5 else 0.0
            pads.append(p)
            nets.setdefault(net, {"name": net if rng.random() < 0.8 else f"{net}_alias", "code": n, "pads": []})
            nets[net]["pads"].append(p)
    bd = {"filename": f"board{seed}.kicad_pcb", "layers": nz, "pads": pads, "nets": nets}
    if rng.random() < 0.7:
        bd["layer_names"] = names
    if rng.random() < 0.7:
        bd.update(x_min=5.0, y_min=6.0, x_max=45.0, y_max=44.0, width=40.0, height=38.0)
    for k, v in (("grid_resolution", 0.25), ("clearance", 0.15), ("track_width", 0.2), ("via_diameter", 0.45),
                 ("via_drill", 0.2), ("thickness", 1.2), ("min_clearance", 0.08), ("expansion_margin", 2.0)):
        if rng.random() < 0.5:
            bd[k] = v
    return bd


def random_solution(seed: int):
    rng = np.random.default_rng(seed)
    layers = ["F.Cu", "In1.Cu", "In2.Cu", "B.Cu"]
    tracks, vias, metrics = [], [], []
    for i in range(int(rng.integers(3, 12))):
        x1, y1, x2, y2 = (round(float(v), 3) for v in 50 * rng.random(4))
        net = f"N{int(rng.integers(0, 5))}"
        style = int(rng.integers(0, 4))
        if style == 0:
            t = {"net": net, "layer": str(rng.choice(layers)), "x1": x1, "y1": y1, "x2": x2, "y2": y2}
        elif style == 1:
            t = {"net_id": net, "layer": str(rng.choice(layers)), "start": (x1, y1), "end": (x2, y2)}
        elif style == 2:
            t = {"net_id": net, "start_x": x1, "start_y": y1, "end_x": x2, "end_y": y2}
        else:
            t = {"layer": str(rng.choice(layers)), "x1": x1, "y1": y1, "x2": x2, "y2": y2}
        if rng.random() < 0.6:
            t["width"] = float(rng.choice([0.15, 0.24]))
        tracks.append(t)
    for i in range(int(rng.integers(1, 8))):
        x, y = (round(float(v), 3) for v in 50 * rng.random(2))
        style = int(rng.integers(0, 4))
        if style == 0:
            v = {"net": f"N{i}", "x": x, "y": y, "from_layer": "F.Cu", "to_layer": "In1.Cu"}
        elif style == 1:
            v = {"net_id": f"N{i}", "position": (x, y), "from_layer": "In1.Cu", "to_layer": "B.Cu"}
        elif style == 2:
            v = {"net_id": f"N{i}", "position": {"x": x, "y": y}}
        else:
            v = {"net": f"N{i}"}
        if rng.random() < 0.5:
            v["drill"] = 0.2
        if rng.random() < 0.5:
            v["size" if rng.random() < 0.5 else "diameter"] = 0.45
        vias.append(v)
    for it in range(int(rng.integers(0, 5))):
        m = {"iteration": it + 1}
        for k in rng.permutation(["overuse", "overuse_count", "nets_routed", "routed", "overflow", "overflow_cost",
                                  "wirelength", "via_count", "vias", "iteration_time", "time"])[:4]:
            m[str(k)] = float(rng.integers(0, 50))
        metrics.append(m)
    meta = {"board_name": f"b{seed}", "total_time": float(rng.random()), "converged": bool(rng.random() < 0.5)}
    if rng.random() < 0.5:
        meta.update(orthoroute_version="0.3.0", total_iterations=len(metrics), nets_routed=int(rng.integers(0, 9)),
                    notes="random")
    return tracks, vias, metrics, meta


@pytest.mark.parametrize("seed", range(8))
def test_orp_equals_reference_on_random_boards(ref_io, tmp_path, seed):
    from orthoroute_b200.orp import board_data_to_orp, orp_to_board_data, read_orp

    orp_exporter, _ = ref_io
    bd = _json(random_board_data(seed))
    path = tmp_path / f"b{seed}.orp"
    orp_exporter.export_board_to_orp(_json(bd), str(path), compress=True)
    ref_doc = _gz(path)
    ours = board_data_to_orp(bd, filename=path.name, timestamp=ref_doc["metadata"]["export_timestamp"])
    assert _json(ours) == ref_doc
    ref_bd = orp_exporter.convert_orp_to_board_data(orp_exporter.import_board_from_orp(str(path)))
    assert _json(orp_to_board_data(read_orp(path))) == _json(ref_bd)


@pytest.mark.parametrize("seed", range(8))
def test_ors_equals_reference_on_random_solutions(ref_io, tmp_path, seed):
    from orthoroute_b200.ors import ors_to_geometry_payload, read_ors, solution_to_ors

    _, ors_exporter = ref_io
    tracks, vias, metrics, meta = random_solution(seed)

    class Payload:
        pass

    pl = Payload()
    pl.tracks, pl.vias = tracks, vias
    path = tmp_path / f"s{seed}.ors"
    ors_exporter.export_solution_to_ors(pl, metrics, meta, str(path), compress=True)
    ref_doc = _gz(path)
    ours = solution_to_ors(pl, metrics, meta, timestamp=ref_doc["metadata"]["export_timestamp"])
    assert _json(ours) == ref_doc
    ref_geom, ref_meta = ors_exporter.import_solution_from_ors(str(path))
    geom, m2 = read_ors(path)
    assert _json([geom, m2]) == _json([ref_geom, ref_meta])
    a, b = ors_to_geometry_payload(geom), ors_exporter.convert_ors_to_geometry_payload(ref_geom)
    assert _json([a.tracks, a.vias]) == _json([b.tracks, b.vias])
