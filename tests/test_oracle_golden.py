"""The oracle is pinned to golden vectors produced by the reference's own code
(tests/golden/make_golden.py).  CPU only."""
import numpy as np

import oracle as O


def _dijkstra_cases(g):
    lat_arrays = {}
    for name in ("a", "b", "c"):
        lat_arrays[ord(name)] = (g[f"{name}_indptr"], g[f"{name}_indices"], g[f"{name}_cost"])
    for k in range(int(g["ncases"])):
        ip, ix, c = lat_arrays[int(g[f"case{k}_lat"][0])]
        yield k, ip, ix, c, int(g[f"case{k}_src"]), int(g[f"case{k}_dst"]), g[f"case{k}_roi"], g[f"case{k}_path"]


def test_dijkstra_matches_reference_paths(golden):
    g = golden("golden_dijkstra.npz")
    n = 0
    for k, ip, ix, c, s, d, roi, path in _dijkstra_cases(g):
        N = ip.shape[0] - 1
        g2r = np.full(N, -1, dtype=np.int32)
        g2r[roi] = np.arange(len(roi), dtype=np.int32)
        p, dist, parent, _ = O.dijkstra(ip, ix, c, [s], dst=d, roi_map=g2r)
        got = p if len(p) > 1 else np.zeros(0, np.int32)
        assert np.array_equal(got, path), f"case {k}: {got} vs reference {path}"
        n += 1
    assert n == int(g["ncases"])


def test_dijkstra_reference_lattice_duplicate_vias(golden):
    """The reference's own Lattice3D graph (inner planar layers, blind/buried
    vias emitted twice)."""
    g = golden("golden_dijkstra.npz")
    ip, ix, c = g["ref_indptr"], g["ref_indices"], g["ref_cost"]
    for k in range(int(g["nref"])):
        s, d = (int(v) for v in g[f"ref{k}_st"])
        p, *_ = O.dijkstra(ip, ix, c, [s], dst=d)
        got = p if len(p) > 1 else np.zeros(0, np.int32)
        assert np.array_equal(got, g[f"ref{k}_path"])


def test_dijkstra_fractional_costs_agreement(golden):
    """float64 path sums (reference) vs float32 (oracle): report agreement; the
    path costs must agree to float32 rounding even when the paths differ."""
    g = golden("golden_dijkstra_frac.npz")
    ip, ix, c = g["indptr"], g["indices"], g["cost"]
    same = 0
    for i, (s, d) in enumerate(zip(g["src"], g["dst"])):
        p, dist, _, _ = O.dijkstra(ip, ix, c, [int(s)], dst=int(d))
        ref = g[f"path{i}"]
        if np.array_equal(p, ref):
            same += 1
        else:
            e_ref = O.path_to_edges(ip, ix, ref)
            e_got = O.path_to_edges(ip, ix, p)
            assert abs(float(np.sum(c[e_ref].astype(np.float64))) - float(np.sum(c[e_got].astype(np.float64)))) < 1e-3
    assert same >= 0.9 * len(g["src"])


def test_roi_bfs_matches_reference(golden):
    g = golden("golden_roi.npz")
    ip, ix = g["indptr"], g["indices"]
    for k in range(int(g["ncases"])):
        s, d, depth, max_nodes = (int(v) for v in g[f"c{k}_args"])
        roi, g2r = O.roi_bfs(ip, ix, s, d, min(depth, 150), max_nodes)
        assert np.array_equal(roi, g[f"c{k}_roi"]), f"case {k}"
        assert np.array_equal(g2r[roi], np.arange(len(roi)))


def test_path_to_edges_matches_reference(golden):
    g = golden("golden_path_edges.npz")
    d = golden("golden_dijkstra.npz")
    ip, ix = d["ref_indptr"], d["ref_indices"]
    for k in range(int(g["n"])):
        got = O.path_to_edges(ip, ix, g[f"p{k}"])
        assert np.array_equal(got, g[f"e{k}"])


def test_accounting_restatements_match_reference(golden):
    g = golden("golden_accounting.npz")
    for i, row in enumerate(g["cost_params"]):
        pf, hw, vm, bw, jit, ub = row
        out = O.update_costs(g["base"], g["ema"], g["cap"], g["hist"], float(pf), float(hw), add_jitter=bool(jit),
                             via_cost_multiplier=float(vm), base_cost_weight=float(bw),
                             edge_layer=g["edge_layer"] if ub else None,
                             layer_bias_per_layer=g["layer_bias"] if ub else None,
                             edge_kind=g["edge_kind"] if ub else None)
        assert out.dtype == np.float32
        assert np.array_equal(out.view(np.uint32), g[f"cost{i}"].view(np.uint32))
    for i, row in enumerate(g["hist_params"]):
        gain, capm, decay, use_base = row
        out = O.update_history(g["hist"], g["present"], g["cap"], float(gain),
                               base_costs=g["base"] if use_base else None, history_cap_multiplier=float(capm),
                               decay_factor=float(decay))
        assert np.array_equal(out.view(np.uint32), g[f"hist{i}"].view(np.uint32))
    ema = O.update_present_ema(g["present"], g["ema"], beta=0.40)
    assert np.array_equal(ema.view(np.uint32), g["ema_out"].view(np.uint32))
    assert tuple(O.compute_overuse(g["over_present"], g["cap"])) == tuple(g["overuse"])


def test_jitter_rounding_beyond_2_24():
    """numpy's float32 arange rounds the index to float32; the kernels use
    fmodf((float)i, 9973) * 1e-6f, which must agree past 2^24 edges."""
    E = (1 << 24) + 3000
    i = np.arange(E - 4000, E, dtype=np.int64)
    a = np.arange(E, dtype=np.float32)[E - 4000:] % 9973 * np.float32(1e-6)
    fi = i.astype(np.float32)
    b = np.fmod(fi, np.float32(9973)) * np.float32(1e-6)
    assert np.array_equal(a.view(np.uint32), b.astype(np.float32).view(np.uint32))


def _via_meta(golden):
    g = golden("golden_via.npz")
    d = golden("golden_dijkstra.npz")
    nx, ny, nz = (int(v) for v in g["via_dims"])
    meta = O.via_edge_metadata(d["ref_indptr"], d["ref_indices"], nx, ny, nz)
    return g, d, (nx, ny, nz), meta


def test_via_usage_matches_reference(golden):
    g, _, (nx, ny, nz), _ = _via_meta(golden)
    col = np.zeros((nx, ny), np.int64)
    seg = np.zeros((nx, ny, nz - 2), np.int64)
    O.via_usage([g[f"vpath{i}"] for i in range(int(g["npaths"]))], nx, ny, nz, col, seg)
    assert np.array_equal(col, g["col_use"]) and np.array_equal(seg, g["seg_use"])


def test_via_penalties_and_hard_block_match_reference(golden):
    g, _, (nx, ny, nz), meta = _via_meta(golden)
    for tag in ("f32", "f64"):
        out = O.via_penalties(g["total0"], meta, g["col_pres"], g["seg_prefix"], nz - 2, g[f"bias_{tag}"], 2.25)
        assert np.array_equal(out.view(np.uint32), g[f"pen_{tag}"].view(np.uint32)), tag
    out = O.via_hard_block(g["total0"], meta, g["col_use"], g["col_cap"], g["seg_use"], g["seg_cap"], nz - 2)
    assert np.array_equal(out.view(np.uint32), g["blocked"].view(np.uint32))
    assert np.isinf(out).sum() > 0
