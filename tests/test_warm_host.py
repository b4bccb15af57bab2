"""Host side of the warm start (no GPU): features, node targets and the
mapping of node predictions back to per-edge history."""
import numpy as np

from orthoroute_b200.lattice import board_footprints
from orthoroute_b200.warm import board_features, history_from_prediction, node_targets


def test_features_targets_and_history_mapping():
    b = board_footprints(64, 64, 6, 30, None, seed=4)
    lat = b.lattice
    f = board_features(lat, b.src, b.dst)
    assert f.shape == (6, 64, 64, 16) and f.dtype == np.float32
    assert f[0, :, :, 0].sum() == 2 * len(b.src)  # every pin once, on the pin layer
    assert f[1:, :, :, 0].sum() == 0
    assert (f[..., 8:] == 0).all()
    # channel 7 (feature set 2): log1p of the RUDY density, the same on every layer
    assert f[..., 7].max() > 0 and np.array_equal(f[0, :, :, 7], f[-1, :, :, 7])
    assert (board_features(lat, b.src, b.dst, version=1)[..., 7:] == 0).all()
    assert f[..., 4].sum() > 0 and f[..., 5].sum() > 0
    rng = np.random.default_rng(0)
    hist = np.zeros(lat.E, np.float32)
    kind = np.asarray(lat.edge_kind)
    # constant history per (node, kind) maps back exactly
    es = lat.edge_src()
    per_node = rng.random((lat.N, 2)).astype(np.float32) * 3
    hist[:] = per_node[es, kind]
    t = node_targets(lat, hist)
    assert t.shape == (6, 64, 64, 2)
    back = history_from_prediction(lat, t, 1.0)
    assert np.allclose(back, hist, rtol=1e-5, atol=1e-5)
    assert np.allclose(history_from_prediction(lat, t, 0.5), 0.5 * hist, rtol=1e-5, atol=1e-5)
