"""Negotiation bookkeeping against golden vectors from the reference's own
methods (tests/golden/make_golden_bookkeeping.py): the oracle restatement
(CPU) and the device kernels (GPU), each followed by the same host selection
logic (orthoroute_b200.bookkeeping)."""
import random

import numpy as np
import pytest

import oracle.bookkeeping as OB
from orthoroute_b200.bookkeeping import difficulty_order, select_hotset
from orthoroute_b200.lattice import board_uniform_pins


def _case(g, c):
    p = f"c{c}_"
    nx, ny, nz, nets, seed = (int(v) for v in g[p + "board"])
    b = board_uniform_pins(nx, ny, nz, nets, seed=seed)
    names = [f"N{k}" for k in range(nets)]
    order = [names[k] for k in g[p + "order"]]
    po = np.concatenate([[0], np.cumsum(g[p + "plen"])])
    eo = np.concatenate([[0], np.cumsum(g[p + "elen"])])
    paths = {n: g[p + "paths"][po[i]:po[i + 1]].tolist() for i, n in enumerate(order)}
    edges = {n: g[p + "edges"][eo[i]:eo[i + 1]].tolist() for i, n in enumerate(order)}
    tasks = {names[k]: (int(b.src[k]), int(b.dst[k])) for k in range(nets)}
    ids = {names[k]: int(g[p + "net_ids"][k]) for k in range(nets)}
    keep = [(int(z), int(x), int(y), names[int(k)]) for z, x, y, k in g[p + "keepouts"]]
    return b, names, order, paths, edges, tasks, ids, keep


def _hot_state(g, c, names):
    p = f"c{c}_"
    clean = {n: int(v) for n, v in zip(names, g[p + "hot_clean_before"])}
    last = {n: int(v) for n, v in zip(names, g[p + "hot_last_before"]) if v != -999}
    return int(g[p + "hot_iteration"]), clean, last, int(g[p + "hot_cap"])


@pytest.mark.parametrize("c", [0, 1])
def test_oracle_bookkeeping_matches_reference(golden, c):
    g = golden("golden_bookkeeping.npz")
    p = f"c{c}_"
    b, names, order, paths, edges, tasks, ids, keep = _case(g, c)
    lat = b.lattice
    owner = OB.node_owner(lat.N, lat.nx, lat.ny, [paths[n] for n in order], [ids[n] for n in order],
                          [(z, x, y, ids[n]) for z, x, y, n in keep])
    assert np.array_equal(owner, g[p + "node_owner"])
    conf, cnt = OB.barrel_conflicts(lat.indptr, lat.indices, [edges[n] for n in order], [ids[n] for n in order],
                                    owner)
    assert cnt == int(g[p + "conflict_count"])
    assert np.array_equal(conf, g[p + "conflicts"])
    after = OB.barrel_penalty(g[p + "present"], conf, float(g[p + "pres_fac"]))
    assert np.array_equal(after.view(np.uint32), g[p + "present_after"].view(np.uint32))
    cong, imp, off, hot = OB.net_scores([edges[n] for n in order], g[p + "present"], g[p + "capacity"],
                                        g[p + "history"])
    random.seed(int(g[p + "shuffle_seed"]))
    got = difficulty_order(tasks, dict(zip(order, cong)), lat.nx, lat.ny)
    assert [names.index(n) for n in got] == g[p + "difficulty_order"].tolist()
    it, clean, last, cap = _hot_state(g, c, names)
    hs = select_hotset(tasks, order, imp, off, hot, {n for n in order if len(paths[n]) > 0}, it, clean, last, cap,
                       ripped={names[1]})
    assert sorted(names.index(n) for n in hs) == g[p + "hotset"].tolist()
    assert [clean[n] for n in names] == g[p + "hot_clean_after"].tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("c", [0, 1])
def test_device_bookkeeping_matches_reference(golden, c):
    import torch

    from orthoroute_b200.bookkeeping import Bookkeeper, apply_barrel_penalty, build_hotset, net_scores
    from orthoroute_b200.solver import DeviceGraph

    g = golden("golden_bookkeeping.npz")
    p = f"c{c}_"
    b, names, order, paths, edges, tasks, ids, keep = _case(g, c)
    lat = b.lattice
    dg = DeviceGraph.from_lattice(lat)
    bk = Bookkeeper(dg)
    owner = bk.rebuild_node_owner(paths, keep).cpu().numpy()
    assert [bk.net_id_map[n] for n in order] == [ids[n] for n in order]
    assert np.array_equal(owner, g[p + "node_owner"])
    mask, cnt = bk.detect_barrel_conflicts(edges)
    assert cnt == int(g[p + "conflict_count"])
    ref_mask = np.zeros(lat.E, bool)
    ref_mask[g[p + "conflicts"]] = True
    assert np.array_equal(mask.cpu().numpy().astype(bool), ref_mask)
    present = torch.from_numpy(g[p + "present"].copy()).cuda()
    apply_barrel_penalty(present, mask, float(g[p + "pres_fac"]))
    assert np.array_equal(present.cpu().numpy().view(np.uint32), g[p + "present_after"].view(np.uint32))
    pres0 = torch.from_numpy(g[p + "present"].copy()).cuda()
    capd = torch.from_numpy(g[p + "capacity"].copy()).cuda()
    histd = torch.from_numpy(g[p + "history"].copy()).cuda()
    cong, imp, off, hot = net_scores(dg, [edges[n] for n in order], pres0, capd, histd)
    rc, ri, ro, rh = OB.net_scores([edges[n] for n in order], g[p + "present"], g[p + "capacity"], g[p + "history"])
    assert np.array_equal(cong.view(np.uint64), rc.view(np.uint64))
    assert np.array_equal(imp.view(np.uint64), ri.view(np.uint64))
    assert np.array_equal(off, ro) and hot == rh
    it, clean, last, cap = _hot_state(g, c, names)
    hs = build_hotset(dg, tasks, edges, {n for n in order if len(paths[n]) > 0}, pres0, capd, histd, it, clean,
                      last, cap, ripped={names[1]})
    assert sorted(names.index(n) for n in hs) == g[p + "hotset"].tolist()


def _golden_geometry(g, c, names):
    p = f"c{c}_"
    ln = [str(v) for v in g[p + "layer_names"]]
    tracks = [(names[int(n)], int(l), tuple(float(v) for v in xy)) for (n, l), xy in zip(g[p + "tracks"],
                                                                                       g[p + "track_xy"])]
    vias = [(names[int(n)], int(a), int(b), tuple(float(v) for v in xy)) for (n, a, b), xy in zip(g[p + "vias"],
                                                                                                 g[p + "via_xy"])]
    return ln, [str(v) for v in g[p + "layer_dir"]], tuple(float(v) for v in g[p + "geom"]), tracks, vias


@pytest.mark.parametrize("c", [0, 1])
def test_oracle_geometry_matches_reference(golden, c):
    import oracle.geometry as OG
    from orthoroute_b200.geometry import _quantize

    g = golden("golden_bookkeeping.npz")
    b, names, order, paths, edges, tasks, ids, keep = _case(g, c)
    lat = b.lattice
    ln, dirs, (gx, gy, pitch), tracks, vias = _golden_geometry(g, c, names)
    out = OG.emit([paths[n] for n in order], lat.nx, lat.ny, lat.nz, dirs)
    plane = lat.nx * lat.ny

    def xy(node):
        r = node % plane
        return (float(_quantize(gx + (r % lat.nx) * pitch, gx, pitch)),
                float(_quantize(gy + (r // lat.nx) * pitch, gy, pitch)))

    got_t, got_v = [], []
    for n, (tr, vi) in zip(order, out):
        got_t += [(n, z, xy(a) + xy(bb)) for a, bb, z in tr]
        got_v += [(n, min(z0, z1), max(z0, z1), xy(v)) for v, z0, z1 in vi]
    assert got_t == tracks
    assert got_v == vias


@pytest.mark.gpu
@pytest.mark.parametrize("c", [0, 1])
def test_device_geometry_matches_reference(golden, c):
    from orthoroute_b200.geometry import generate_geometry
    from orthoroute_b200.solver import DeviceGraph

    g = golden("golden_bookkeeping.npz")
    b, names, order, paths, edges, tasks, ids, keep = _case(g, c)
    ln, dirs, (gx, gy, pitch), tracks, vias = _golden_geometry(g, c, names)
    dg = DeviceGraph.from_lattice(b.lattice)
    t, v = generate_geometry(dg, paths, dirs, gx, gy, pitch, ln, grid_pitch=pitch)
    assert [(d["net"], ln.index(d["layer"]), (d["x1"], d["y1"], d["x2"], d["y2"])) for d in t] == tracks
    assert [(d["net"], ln.index(d["from_layer"]), ln.index(d["to_layer"]), (d["x"], d["y"])) for d in v] == vias
