"""Learned history warm start for PathFinder.

A small 3D convolutional net predicts, from the pins and the airwires of a
board, the history cost field PathFinder ends with; routing then starts from
that history instead of zero.  Plain zero-history PathFinder stays both the
fallback and the yardstick: a warm run counts only when it reaches zero
overuse, and if it has not converged within 1.5x the plain run's iterations
the plain run is used.

Network (all layers run by the kernels of orsp_warm.cu, bf16 activations
[D][H][W][C] with fp32 accumulation): a 4-level U-net over the routing grid,
32 channels at every level, two 3x3x3 convolutions + ReLU per encoder level,
2x2 average pooling in x/y between levels (the layer count is small and is
kept), nearest upsampling + skip addition + one convolution per decoder
level, and a 3x3x3 head with 16 output channels of which two are used: the
mean history of a node's planar out-edges and of its via out-edges,
predicted as log1p(history).

Inputs per cell (16 channels, unused ones zero): pin density on the pin
layer, blurred pin density, airwire (pin-to-pin segment) crossing density,
net bounding-box coverage, H-layer flag, V-layer flag, layer position.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr
from .lattice import Lattice, layer_directions

F_IN = 16   # input channels (padded)
F_OUT = 16  # head channels (2 used)
USED = 2


def _st() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


# ----------------------------------------------------------------- features
def _box_blur(a: np.ndarray, r: int) -> np.ndarray:
    """Mean over a (2r+1)^2 window (edges: smaller window), float32."""
    c = np.pad(a.astype(np.float64), ((1, 0), (1, 0))).cumsum(0).cumsum(1)
    H, W = a.shape
    y0 = np.clip(np.arange(H) - r, 0, H)
    y1 = np.clip(np.arange(H) + r + 1, 0, H)
    x0 = np.clip(np.arange(W) - r, 0, W)
    x1 = np.clip(np.arange(W) + r + 1, 0, W)
    s = c[y1][:, x1] - c[y0][:, x1] - c[y1][:, x0] + c[y0][:, x0]
    n = (y1 - y0)[:, None] * (x1 - x0)[None, :]
    return (s / n).astype(np.float32)


FEATURES = 2  # feature set of newly built networks (see board_features)


def _segment_points(a, b, c, d):
    """The cells of every pin-to-pin segment rasterised at unit steps, as
    np.rint(np.linspace(a, c, n)) and np.rint(np.linspace(b, d, n)) with
    n = max(|c - a|, |d - b|) + 1 give them per segment (linspace's
    k * step + start, its exact end point), for all segments at once."""
    a, b, c, d = (np.asarray(v, np.int64) for v in (a, b, c, d))
    n = np.maximum(np.abs(c - a), np.abs(d - b)) + 1
    seg = np.repeat(np.arange(n.size), n)
    k = np.arange(seg.size) - np.repeat(np.cumsum(n) - n, n)
    div = np.maximum(n - 1, 1).astype(np.float64)

    def coord(p, q):
        step = (q - p).astype(np.float64) / div
        y = k.astype(np.float64) * step[seg] + p[seg].astype(np.float64)
        last = (k == n[seg] - 1) & (n[seg] > 1)
        y[last] = q[seg][last]
        return np.rint(y).astype(np.int64)

    return coord(a, c), coord(b, d)


def _air_counts_device(sx, sy, dx, dy, nx: int, ny: int, device) -> np.ndarray:
    """The airwire crossing counts of _segment_points, float32 [ny][nx], with
    the rasterisation on `device`: the same float64 operations (one division,
    one multiply, one add, each rounded once), linspace's exact end point and
    round-half-even, so the same cells as on the host; counts are integers."""
    dev = torch.device(device)
    a, b, c, d = (torch.from_numpy(np.ascontiguousarray(v, dtype=np.int64)).to(dev) for v in (sx, sy, dx, dy))
    n = torch.maximum((c - a).abs(), (d - b).abs()) + 1
    seg = torch.repeat_interleave(torch.arange(n.numel(), device=dev), n)
    start = torch.cumsum(n, 0) - n
    k = torch.arange(seg.numel(), device=dev) - start[seg]
    div = torch.clamp(n - 1, min=1).double()
    ns = n[seg]
    last = (k == ns - 1) & (ns > 1)

    def coord(p, q):
        step = (q - p).double() / div
        y = k.double() * step[seg]
        y = y + p[seg].double()
        y = torch.where(last, q[seg].double(), y)
        return torch.round(y).long()

    cell = coord(b, d) * nx + coord(a, c)
    return torch.bincount(cell, minlength=ny * nx).to(torch.float32).reshape(ny, nx).cpu().numpy()


def board_maps(lat: Lattice, src: np.ndarray, dst: np.ndarray, version: int = FEATURES, device=None) -> dict:
    """The board-dependent 2-D maps of board_features (host, float32 [ny][nx]),
    the pin layer, and the layer flags; with `device`, the airwire
    rasterisation runs there (the same cells)."""
    nx, ny, nz = lat.nx, lat.ny, lat.nz
    sx, sy, sz = (np.asarray(v) for v in lat.coords(np.asarray(src)))
    dx, dy, dz = (np.asarray(v) for v in lat.coords(np.asarray(dst)))
    pins = np.zeros((ny, nx), np.float32)
    np.add.at(pins, (sy, sx), 1.0)
    np.add.at(pins, (dy, dx), 1.0)
    # airwire crossing density: each pin-to-pin segment rasterised at unit steps
    # (integer counts, exact in float32)
    if device is not None:
        air = _air_counts_device(sx, sy, dx, dy, nx, ny, device)
    else:
        xs, ys = _segment_points(sx, sy, dx, dy)
        air = np.bincount(ys * nx + xs, minlength=ny * nx).astype(np.float32).reshape(ny, nx)
    cov = np.zeros((ny + 1, nx + 1), np.float32)
    x0, x1 = np.minimum(sx, dx), np.maximum(sx, dx) + 1
    y0, y1 = np.minimum(sy, dy), np.maximum(sy, dy) + 1
    np.add.at(cov, (y0, x0), 1.0)
    np.add.at(cov, (y0, x1), -1.0)
    np.add.at(cov, (y1, x0), -1.0)
    np.add.at(cov, (y1, x1), 1.0)
    cov = cov.cumsum(0).cumsum(1)[:ny, :nx]
    m = {"pin_layer": int(np.bincount(np.concatenate([sz, dz]).astype(np.int64), minlength=nz).argmax()),
         "pins": pins, "pin_blur": _box_blur(pins, 4) * 4.0, "air": _box_blur(air, 2) / 8.0, "cov": cov / 32.0,
         "dirs": layer_directions(nz)}
    if version >= 2:
        m["rudy"] = np.log1p(rudy_density(lat, src, dst)).astype(np.float32)
    return m


def board_features(lat: Lattice, src: np.ndarray, dst: np.ndarray, version: int = FEATURES) -> np.ndarray:
    """float32 [nz][ny][nx][16] input features of a board (host).  Channels:
    0 pins on the pin layer, 1 blurred pin density, 2 airwire crossing density,
    3 bounding-box coverage, 4 / 5 H / V layer, 6 layer position; version 2
    adds 7, log1p of the RUDY wire density (rudy_density)."""
    nx, ny, nz = lat.nx, lat.ny, lat.nz
    m = board_maps(lat, src, dst, version)
    f = np.zeros((nz, ny, nx, F_IN), np.float32)
    f[m["pin_layer"], :, :, 0] = m["pins"]
    f[:, :, :, 1] = m["pin_blur"][None]
    f[:, :, :, 2] = m["air"][None]
    f[:, :, :, 3] = m["cov"][None]
    for z, d in enumerate(m["dirs"]):
        f[z, :, :, 4] = 1.0 if "h" in d else 0.0
        f[z, :, :, 5] = 1.0 if "v" in d else 0.0
        f[z, :, :, 6] = z / max(1, nz - 1)
    if version >= 2:
        f[:, :, :, 7] = m["rudy"][None]
    return f


def board_features_device(lat: Lattice, src, dst, version: int = FEATURES, device=None) -> torch.Tensor:
    """board_features assembled on the device, as the network reads it: bf16
    [nz][H8][W8][16] with H, W padded to multiples of 8 with zeros.  The 2-D
    maps come from board_maps (host, float32), so every value equals the
    host array's after the same bf16 conversion."""
    dev = torch.device(device) if device is not None else torch.device("cuda")
    nx, ny, nz = lat.nx, lat.ny, lat.nz
    m = board_maps(lat, src, dst, version, device=dev)
    Hp, Wp = (ny + 7) // 8 * 8, (nx + 7) // 8 * 8
    f = torch.zeros((nz, Hp, Wp, F_IN), dtype=torch.float32, device=dev)
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    f[m["pin_layer"], :ny, :nx, 0] = up(m["pins"])
    f[:, :ny, :nx, 1] = up(m["pin_blur"])[None]
    f[:, :ny, :nx, 2] = up(m["air"])[None]
    f[:, :ny, :nx, 3] = up(m["cov"])[None]
    for z, d in enumerate(m["dirs"]):
        f[z, :ny, :nx, 4] = 1.0 if "h" in d else 0.0
        f[z, :ny, :nx, 5] = 1.0 if "v" in d else 0.0
        f[z, :ny, :nx, 6] = z / max(1, nz - 1)
    if version >= 2:
        f[:, :ny, :nx, 7] = up(m["rudy"])[None]
    return f.to(torch.bfloat16)


def node_targets(lat: Lattice, history: np.ndarray, blur: int = 0) -> np.ndarray:
    """float32 [nz][ny][nx][2]: log1p of the mean history of each node's planar
    and via out-edges (0 where it has none), optionally averaged over a
    (2 blur + 1)^2 window in x/y (a smooth congestion map)."""
    # per (node, kind) sums in edge order
    idx = lat.edge_src().astype(np.int64) * 2 + np.asarray(lat.edge_kind).astype(np.int64)
    out = np.bincount(idx, weights=np.asarray(history, np.float64), minlength=2 * lat.N).reshape(lat.N, 2)
    cnt = np.bincount(idx, minlength=2 * lat.N).astype(np.float64).reshape(lat.N, 2)
    mean = np.where(cnt > 0, out / np.maximum(cnt, 1), 0.0)
    t = np.log1p(mean).astype(np.float32).reshape(lat.nz, lat.ny, lat.nx, 2)
    if blur > 0:
        for z in range(lat.nz):
            for c in range(2):
                t[z, :, :, c] = _box_blur(t[z, :, :, c], blur)
    return t


def history_from_prediction(lat: Lattice, pred: np.ndarray, scale: float = 1.0) -> np.ndarray:
    """Per-edge history (float32[E]) from node predictions [nz][ny][nx][2]:
    every out-edge of a node gets expm1 of its kind's channel, times scale."""
    p = np.expm1(np.maximum(pred.reshape(lat.N, 2).astype(np.float64), 0.0))
    kind = np.asarray(lat.edge_kind).astype(np.int64)
    return (p[lat.edge_src(), kind] * scale).astype(np.float32)


def rudy_density(lat: Lattice, src: np.ndarray, dst: np.ndarray) -> np.ndarray:
    """RUDY wire density per cell and routing layer, float64 [ny][nx]: each
    net's half-perimeter wire length (w + h) spread uniformly over its bounding
    box (w x h cells), summed over nets, divided by the layer count."""
    nx, ny, nz = lat.nx, lat.ny, lat.nz
    sx, sy, _ = (np.asarray(v).astype(np.int64) for v in lat.coords(np.asarray(src)))
    dx, dy, _ = (np.asarray(v).astype(np.int64) for v in lat.coords(np.asarray(dst)))
    x0, x1 = np.minimum(sx, dx), np.maximum(sx, dx) + 1
    y0, y1 = np.minimum(sy, dy), np.maximum(sy, dy) + 1
    w = (x1 - x0).astype(np.float64)
    h = (y1 - y0).astype(np.float64)
    dens = (w + h) / (w * h)
    acc = np.zeros((ny + 1, nx + 1), np.float64)
    np.add.at(acc, (y0, x0), dens)
    np.add.at(acc, (y0, x1), -dens)
    np.add.at(acc, (y1, x0), -dens)
    np.add.at(acc, (y1, x1), dens)
    return np.maximum(acc.cumsum(0).cumsum(1)[:ny, :nx] / nz, 0.0)


def rudy_prediction(lat: Lattice, src: np.ndarray, dst: np.ndarray) -> np.ndarray:
    """A non-learned congestion prior in the network's output format
    ([nz][ny][nx][2], log1p domain): log1p of the RUDY density
    (rudy_density), the same on every layer and edge kind.  It is the
    baseline the learned prediction is compared with: the same history
    mapping and scale search apply to both."""
    p = np.log1p(rudy_density(lat, src, dst)).astype(np.float32)
    out = np.empty((lat.nz, lat.ny, lat.nx, 2), np.float32)
    out[:] = p[None, :, :, None]
    return out


# ----------------------------------------------------------------- the net
@dataclass
class Layer:
    name: str
    cin: int
    cout: int
    relu: bool


def architecture(C: int = 32) -> List[Layer]:
    L = [Layer("e0a", F_IN, C, True), Layer("e0b", C, C, True),
         Layer("e1a", C, C, True), Layer("e1b", C, C, True),
         Layer("e2a", C, C, True), Layer("e2b", C, C, True),
         Layer("e3a", C, C, True), Layer("e3b", C, C, True),
         Layer("d2", C, C, True), Layer("d1", C, C, True), Layer("d0", C, C, True),
         Layer("head", C, F_OUT, False)]
    return L


class WarmNet:
    """The U-net, its fp32 master weights and Adam state, on one GPU."""

    def __init__(self, C: int = 32, device=None, seed: int = 0):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.C = C
        self.layers = architecture(C)
        g = torch.Generator().manual_seed(seed)
        self.w: Dict[str, torch.Tensor] = {}
        self.b: Dict[str, torch.Tensor] = {}
        for l in self.layers:
            std = math.sqrt(2.0 / (27 * l.cin)) if l.relu else math.sqrt(1.0 / (27 * l.cin))
            self.w[l.name] = (torch.randn(27, l.cin, l.cout, generator=g) * std).to(self.device)
            self.b[l.name] = torch.zeros(l.cout, device=self.device)
        self.m = {k: torch.zeros_like(v) for k, v in list(self.w.items()) + [("b_" + k, v) for k, v in self.b.items()]}
        self.v = {k: torch.zeros_like(v) for k, v in self.m.items()}
        self.t = 0
        self._packed: Dict[str, torch.Tensor] = {}
        # convolution kernel: "tc" (tcgen05.mma with a TMEM accumulator,
        # orsp_warm_conv3d_tc) or "wmma" (orsp_warm_conv3d); ORSP_WARM_CONV
        # overrides the default
        self.conv_impl = os.environ.get("ORSP_WARM_CONV", "tc")
        self.features = FEATURES  # input feature set (board_features version)

    def _conv_call(self, *args):
        lib = _lib.load()
        if self.conv_impl == "tc":
            return check(lib.orsp_warm_conv3d_tc(*args), "orsp_warm_conv3d_tc")
        return check(lib.orsp_warm_conv3d(*args), "orsp_warm_conv3d")

    # weights as the conv kernel reads them
    def _pack(self, name: str, transpose: bool) -> torch.Tensor:
        l = next(x for x in self.layers if x.name == name)
        key = name + ("/T" if transpose else "")
        out = self._packed.get(key)
        if out is None:
            out = torch.empty(27 * l.cin * l.cout, dtype=torch.bfloat16, device=self.device)
            self._packed[key] = out
        check(_lib.load().orsp_warm_pack_weights(ptr(self.w[name]), ptr(out), l.cin, l.cout, 1 if transpose else 0,
                                                 _st()), "orsp_warm_pack_weights")
        return out

    def _conv(self, x, name, D, H, W, out_f32=False):
        l = next(y for y in self.layers if y.name == name)
        if out_f32:
            y = torch.empty(D, H, W, l.cout, dtype=torch.float32, device=self.device)
            yb, yf = None, y
        else:
            y = torch.empty(D, H, W, l.cout, dtype=torch.bfloat16, device=self.device)
            yb, yf = y, None
        self._conv_call(ptr(x), None, ptr(self._packed[name]), ptr(self.b[name]), ptr(yb), ptr(yf), D, H, W, l.cin,
                        l.cout, 1 if l.relu else 0, _st())
        return y

    def _pool(self, x, D, H, W):
        y = torch.empty(D, H // 2, W // 2, x.shape[-1], dtype=torch.bfloat16, device=self.device)
        check(_lib.load().orsp_warm_pool(ptr(x), ptr(y), D, H, W, x.shape[-1], _st()), "orsp_warm_pool")
        return y

    def _spread(self, xc, D, H, W, scale):
        y = torch.empty(D, H, W, xc.shape[-1], dtype=torch.bfloat16, device=self.device)
        check(_lib.load().orsp_warm_spread(ptr(xc), ptr(y), D, H, W, xc.shape[-1], float(scale), _st()),
              "orsp_warm_spread")
        return y

    def _gather4(self, xf, D, H, W):
        y = torch.empty(D, H // 2, W // 2, xf.shape[-1], dtype=torch.bfloat16, device=self.device)
        check(_lib.load().orsp_warm_gather4(ptr(xf), ptr(y), D, H, W, xf.shape[-1], _st()), "orsp_warm_gather4")
        return y

    def _add(self, a, b):
        y = torch.empty_like(a)
        check(_lib.load().orsp_warm_add(ptr(a), ptr(b), ptr(y), a.numel(), _st()), "orsp_warm_add")
        return y

    # -------------------------------------------------------------- forward
    def forward(self, x: torch.Tensor, keep: bool = False):
        """x: bf16 [D][H][W][16], H and W multiples of 8.  Returns the fp32
        head output [D][H][W][16] (and the activations when keep)."""
        D, H, W = x.shape[:3]
        if H % 8 or W % 8:
            raise ValueError("warm net: H and W must be multiples of 8")
        for l in self.layers:
            self._pack(l.name, False)
        a = {"x": x}
        dims = [(D, H, W), (D, H // 2, W // 2), (D, H // 4, W // 4), (D, H // 8, W // 8)]
        h = x
        for lev in range(4):
            d = dims[lev]
            if lev > 0:
                h = self._pool(a[f"e{lev - 1}b"], *dims[lev - 1])
                a[f"p{lev}"] = h
            a[f"e{lev}a"] = self._conv(h, f"e{lev}a", *d)
            a[f"e{lev}b"] = self._conv(a[f"e{lev}a"], f"e{lev}b", *d)
        h = a["e3b"]
        for lev in (2, 1, 0):
            d = dims[lev]
            up = self._spread(h, *d, 1.0)
            a[f"m{lev}"] = self._add(up, a[f"e{lev}b"])
            h = self._conv(a[f"m{lev}"], f"d{lev}", *d)
            a[f"d{lev}"] = h
        out = self._conv(h, "head", D, H, W, out_f32=True)
        return (out, a) if keep else out

    # ------------------------------------------------------------- backward
    def _conv_back(self, x_in, y_out, dy, name, D, H, W, need_dx=True):
        """Gradients of one conv layer: accumulates dW, db; returns dx."""
        l = next(z for z in self.layers if z.name == name)
        lib = _lib.load()
        mask = y_out if l.relu else None
        wgrad = lib.orsp_warm_wgrad_tc if self.conv_impl == "tc" else lib.orsp_warm_wgrad
        check(wgrad(ptr(x_in), ptr(dy), ptr(mask), ptr(self.gw[name]), ptr(self.gb[name]), D, H, W, l.cin, l.cout,
                    _st()), "orsp_warm_wgrad")
        if not need_dx:
            return None
        wt = self._pack(name, True)
        dx = torch.empty(D, H, W, l.cin, dtype=torch.bfloat16, device=self.device)
        self._conv_call(ptr(dy), ptr(mask), ptr(wt), None, ptr(dx), None, D, H, W, l.cout, l.cin, 0, _st())
        return dx

    def backward(self, a: dict, dout: torch.Tensor):
        """dout: bf16 gradient of the head output [D][H][W][16].  Fills
        self.gw / self.gb (fp32)."""
        self.gw = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.gb = {k: torch.zeros_like(v) for k, v in self.b.items()}
        D, H, W = a["x"].shape[:3]
        dims = [(D, H, W), (D, H // 2, W // 2), (D, H // 4, W // 4), (D, H // 8, W // 8)]
        g = self._conv_back(a["d0"], None, dout, "head", *dims[0])
        skip_g = {}
        for lev in (0, 1, 2):
            d = dims[lev]
            gm = self._conv_back(a[f"m{lev}"], a[f"d{lev}"], g, f"d{lev}", *d)
            skip_g[lev] = gm  # gradient into e{lev}b through the skip addition
            # gradient into the coarser level through the upsampling
            g = self._gather4(gm, *d)
        # bottleneck and encoder
        for lev in (3, 2, 1, 0):
            d = dims[lev]
            ge_b = g if lev == 3 else self._add(g, skip_g[lev])
            ge_a = self._conv_back(a[f"e{lev}a"], a[f"e{lev}b"], ge_b, f"e{lev}b", *d)
            x_in = a["x"] if lev == 0 else a[f"p{lev}"]
            gx = self._conv_back(x_in, a[f"e{lev}a"], ge_a, f"e{lev}a", *d, need_dx=lev > 0)
            if lev > 0:
                g = self._spread(gx, *dims[lev - 1], 0.25)  # adjoint of 2x2 averaging

    def loss_grad(self, out: torch.Tensor, target: torch.Tensor, weight: Optional[torch.Tensor] = None):
        """MSE over the two used channels; returns (loss tensor [1], dout bf16)."""
        D, H, W = out.shape[:3]
        nvox = D * H * W
        dout = torch.empty(D, H, W, F_OUT, dtype=torch.bfloat16, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        check(_lib.load().orsp_warm_mse(ptr(out), ptr(target), ptr(weight), ptr(dout), ptr(loss), nvox, F_OUT, USED,
                                        1.0 / (nvox * USED), _st()), "orsp_warm_mse")
        return loss, dout

    def step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8, wd: float = 0.0):
        self.t += 1
        lr_t = lr * math.sqrt(1 - b2 ** self.t) / (1 - b1 ** self.t)
        lib = _lib.load()
        for k in self.w:
            for p, g, key in ((self.w[k], self.gw[k], k), (self.b[k], self.gb[k], "b_" + k)):
                check(lib.orsp_warm_adam(ptr(p), ptr(g), ptr(self.m[key]), ptr(self.v[key]), p.numel(), float(lr_t),
                                         float(b1), float(b2), float(eps), float(wd), _st()), "orsp_warm_adam")

    # ------------------------------------------------------------ utilities
    def state(self) -> dict:
        out = {}
        for k in self.w:
            out["w_" + k] = self.w[k].cpu().numpy()
            out["b_" + k] = self.b[k].cpu().numpy()
        return out

    def load_state(self, st: dict):
        for k in self.w:
            self.w[k].copy_(torch.from_numpy(np.asarray(st["w_" + k], np.float32)))
            self.b[k].copy_(torch.from_numpy(np.asarray(st["b_" + k], np.float32)))

    def predict(self, feats: np.ndarray) -> np.ndarray:
        """feats float32 [D][H][W][16] (any H, W: padded to multiples of 8 with
        zeros) -> float32 [D][H][W][2] (log1p history per node and kind)."""
        D, H, W = feats.shape[:3]
        Hp, Wp = (H + 7) // 8 * 8, (W + 7) // 8 * 8
        x = np.zeros((D, Hp, Wp, F_IN), np.float32)
        x[:, :H, :W] = feats
        xt = torch.from_numpy(x).to(self.device).to(torch.bfloat16)
        out = self.forward(xt)
        return out[:, :H, :W, :USED].cpu().numpy()


DEFAULT_WEIGHTS = __import__("pathlib").Path(__file__).resolve().parent / "data" / "warm_history.npz"


def load_pretrained(path=None, device=None) -> Tuple["WarmNet", float]:
    """The shipped network (trained by orthoroute_b200.warm_train) and its
    history scale."""
    st = dict(np.load(path or DEFAULT_WEIGHTS))
    net = WarmNet(C=32, device=device)
    net.load_state({k: v.astype(np.float32) for k, v in st.items() if k.startswith(("w_", "b_"))})
    net.features = int(st.get("features", 1))  # files written before version 2 carry no version
    return net, float(st.get("scale", 1.0))


def pretrained_rudy_scale(path=None) -> Optional[float]:
    """The history scale chosen for the RUDY prior on the same held-out
    boards as the network's (None if the shipped file has none)."""
    st = np.load(path or DEFAULT_WEIGHTS)
    return float(st["rudy_scale"]) if "rudy_scale" in st.files else None


def warm_history(net: "WarmNet", lat: Lattice, src, dst, scale: float) -> np.ndarray:
    """Initial per-edge history for a board: features -> net -> edges."""
    pred = net.predict(board_features(lat, np.asarray(src), np.asarray(dst), net.features))
    return history_from_prediction(lat, pred, scale)


def warm_history_device(net: "WarmNet", lat: Lattice, src, dst, scale: float) -> torch.Tensor:
    """warm_history with the feature assembly, the forward pass and the
    node -> edge mapping on the device: float32 [E] (device).  The mapping is
    history_from_prediction's (expm1 of the clamped prediction in float64,
    times scale, rounded to float32)."""
    dev = net.device
    x = board_features_device(lat, np.asarray(src), np.asarray(dst), net.features, device=dev)
    out = net.forward(x)[:, :lat.ny, :lat.nx, :USED].float()
    return history_from_prediction_device(lat, out, scale)


def history_from_prediction_device(lat: Lattice, pred: torch.Tensor, scale: float) -> torch.Tensor:
    """history_from_prediction on the device: pred float32 [nz][ny][nx][2]
    (device) -> float32 [E] (device); expm1 of the clamped prediction in
    float64, times scale, rounded to float32."""
    dev = pred.device
    p = torch.expm1(torch.clamp(pred.reshape(lat.N, 2).double(), min=0.0))
    indptr = torch.from_numpy(np.ascontiguousarray(lat.indptr, dtype=np.int64)).to(dev)
    es = torch.repeat_interleave(torch.arange(lat.N, device=dev), indptr[1:] - indptr[:-1])
    ek = torch.from_numpy(np.ascontiguousarray(lat.edge_kind)).to(dev).long()
    return (p[es, ek] * float(scale)).float()


def _main(argv=None):
    """python -m orthoroute_b200.warm [--size 400] [--nz 18] [--seed 3] [--reps 3]:
    the shipped network's prediction for a footprint board at the backplane's
    net density; prints the time of the features, of one forward pass and of
    its first 3x3x3 convolution (32 -> 32 channels, full resolution) with the
    tensor-core rate that convolution reaches."""
    import argparse
    import json
    import time

    from .lattice import board_footprints

    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=400)
    ap.add_argument("--nz", type=int, default=18)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    nets = int(round(8000 / (600 * 600) * a.size * a.size))
    b = board_footprints(a.size, a.size, a.nz, nets, None, seed=a.seed)
    t0 = time.perf_counter()
    net, scale = load_pretrained()
    feats = board_features(b.lattice, b.src, b.dst, net.features)
    t_feat = time.perf_counter() - t0
    x = torch.from_numpy(feats).cuda().to(torch.bfloat16)
    net.forward(x)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / a.reps
    D, H, W = x.shape[:3]
    h = torch.empty(D, H, W, net.C, dtype=torch.bfloat16, device="cuda").uniform_()
    net._pack("e0b", False)
    e0.record()
    for _ in range(a.reps):
        net._conv(h, "e0b", D, H, W)
    e1.record()
    torch.cuda.synchronize()
    conv_ms = e0.elapsed_time(e1) / a.reps
    flops = 2.0 * 27 * net.C * net.C * D * H * W
    t_hist = {}
    for name, fn in (("host", warm_history), ("device", warm_history_device)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn(net, b.lattice, b.src, b.dst, scale)
        torch.cuda.synchronize()
        t_hist[name] = round(time.perf_counter() - t0, 3)
    print(json.dumps({"board": f"{a.size}x{a.size}x{a.nz}", "voxels": D * H * W, "features_s": round(t_feat, 3),
                      "warm_history_s": t_hist, "forward_ms": round(fwd_ms, 2), "conv32_ms": round(conv_ms, 3),
                      "conv32_tflops": round(flops / (conv_ms / 1e3) / 1e12, 1), "history_scale": scale}))


if __name__ == "__main__":
    _main()
