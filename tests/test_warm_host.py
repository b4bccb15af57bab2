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


def _air_loop(sx, sy, dx, dy, nx, ny):
    air = np.zeros((ny, nx), np.float32)
    for a, b, c, d in zip(sx, sy, dx, dy):
        n = int(max(abs(int(c) - int(a)), abs(int(d) - int(b)))) + 1
        xs = np.rint(np.linspace(a, c, n)).astype(np.int64)
        ys = np.rint(np.linspace(b, d, n)).astype(np.int64)
        air[ys, xs] += 1.0
    return air


def test_segment_rasterisation_matches_linspace():
    """The all-segments rasterisation equals one np.linspace per segment,
    cell for cell, including zero-length segments and ties at .5 steps."""
    from orthoroute_b200.warm import _segment_points

    rng = np.random.default_rng(11)
    nx, ny = 97, 61
    sx, dx = rng.integers(0, nx, 500), rng.integers(0, nx, 500)
    sy, dy = rng.integers(0, ny, 500), rng.integers(0, ny, 500)
    sx[:20], sy[:20] = dx[:20], dy[:20]           # zero length
    sx[20:40], dx[20:40] = 3, 4                   # one-step x, long y
    xs, ys = _segment_points(sx, sy, dx, dy)
    air = np.bincount(ys * nx + xs, minlength=ny * nx).astype(np.float32).reshape(ny, nx)
    assert np.array_equal(air, _air_loop(sx, sy, dx, dy, nx, ny))
    # the torch form the device path runs, here on the CPU
    from orthoroute_b200.warm import _air_counts_device

    assert np.array_equal(_air_counts_device(sx, sy, dx, dy, nx, ny, "cpu"), air)


def test_device_feature_assembly_matches_host_on_cpu():
    """board_features_device, run with device='cpu', equals board_features
    after the bf16 conversion, with zeros in the padding to multiples of 8."""
    import torch

    from orthoroute_b200.warm import board_features_device

    b = board_footprints(83, 45, 6, 60, None, seed=9)
    lat = b.lattice
    f = board_features(lat, b.src, b.dst)
    fd = board_features_device(lat, b.src, b.dst, device="cpu")
    assert fd.shape == (6, 48, 88, 16) and fd.dtype == torch.bfloat16
    assert torch.equal(fd[:, :45, :83], torch.from_numpy(f).to(torch.bfloat16))
    assert float(fd[:, 45:].abs().sum()) == 0 and float(fd[:, :, 83:].abs().sum()) == 0


def test_history_mapping_device_form_on_cpu():
    """history_from_prediction_device (the torch form bench.py and the warm
    route use), run on the CPU, equals history_from_prediction to within one
    float32 ulp (the two expm1 implementations may differ in the last bit),
    with the same edge order."""
    import torch

    from orthoroute_b200.warm import history_from_prediction_device

    b = board_footprints(64, 64, 6, 30, None, seed=7)
    lat = b.lattice
    rng = np.random.default_rng(3)
    pred = (rng.standard_normal((lat.nz, lat.ny, lat.nx, 2)) * 0.7).astype(np.float32)
    host = history_from_prediction(lat, pred, 4.0)
    dev = history_from_prediction_device(lat, torch.from_numpy(pred), 4.0).numpy()
    assert dev.dtype == np.float32 and dev.shape == host.shape
    ulp = np.abs(dev.view(np.int32).astype(np.int64) - host.view(np.int32).astype(np.int64))
    assert int(ulp.max()) <= 1
    assert (host[np.all(pred.reshape(-1, 2)[lat.edge_src()] <= 0, axis=1)] == 0).all()
