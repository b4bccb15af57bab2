"""The warm-start network's CPU oracle (oracle/warm_ref.py) pinned against
central finite differences in float64, and its weight layout against a
direct evaluation of the convolution sum.  CPU only."""
import numpy as np
import torch

from oracle import warm_ref as R


def _params(C=16, seed=0, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    p = {}
    for name, relu in R.LAYERS:
        ci = 16 if name == "e0a" else C
        co = 16 if name == "head" else C
        p[name] = (torch.randn(27, ci, co, generator=g, dtype=dtype) * (0.5 / np.sqrt(27 * ci)),
                   torch.randn(co, generator=g, dtype=dtype) * 0.05 + 0.02)
    return p


def test_conv_layout_matches_direct_sum():
    g = torch.Generator().manual_seed(1)
    x = torch.randn(3, 4, 5, 2, generator=g, dtype=torch.float64)  # [D][H][W][C]
    w = torch.randn(27, 2, 3, generator=g, dtype=torch.float64)
    b = torch.zeros(3, dtype=torch.float64)
    y = R.conv(x.permute(3, 0, 1, 2).unsqueeze(0), w, b, False).squeeze(0).permute(1, 2, 3, 0)
    D, H, W = 3, 4, 5
    ref = torch.zeros(D, H, W, 3, dtype=torch.float64)
    for z in range(D):
        for yy in range(H):
            for xx in range(W):
                for tap in range(27):
                    dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
                    zz, y2, x2 = z + dz, yy + dy, xx + dx
                    if 0 <= zz < D and 0 <= y2 < H and 0 <= x2 < W:
                        ref[z, yy, xx] += x[zz, y2, x2] @ w[tap]
    assert torch.allclose(y, ref, atol=1e-12)


def test_oracle_gradients_match_finite_differences():
    p = _params()
    g = torch.Generator().manual_seed(2)
    x = torch.rand(2, 8, 8, 16, generator=g, dtype=torch.float64)
    t = torch.rand(2, 8, 8, 2, generator=g, dtype=torch.float64)
    _, gr = R.grads(p, x, t, dtype=torch.float64)
    rng = np.random.default_rng(3)
    h = 1e-6
    for name in ("e0a", "e2b", "e3a", "d1", "head"):
        w, b = p[name]
        for _ in range(3):
            i = tuple(int(rng.integers(s)) for s in w.shape)
            wp = {k: (v[0].clone(), v[1].clone()) for k, v in p.items()}
            wm = {k: (v[0].clone(), v[1].clone()) for k, v in p.items()}
            wp[name][0][i] += h
            wm[name][0][i] -= h
            fd = (R.loss_fn(R.forward(wp, x), t) - R.loss_fn(R.forward(wm, x), t)) / (2 * h)
            assert abs(float(fd) - float(gr[name][0][i])) < 1e-6 + 1e-4 * abs(float(fd)), (name, i)
        j = int(rng.integers(b.shape[0]))
        bp = {k: (v[0].clone(), v[1].clone()) for k, v in p.items()}
        bm = {k: (v[0].clone(), v[1].clone()) for k, v in p.items()}
        bp[name][1][j] += h
        bm[name][1][j] -= h
        fd = (R.loss_fn(R.forward(bp, x), t) - R.loss_fn(R.forward(bm, x), t)) / (2 * h)
        assert abs(float(fd) - float(gr[name][1][j])) < 1e-6 + 1e-4 * abs(float(fd)), (name, "bias", j)
