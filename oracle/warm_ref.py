"""ORACLE - test infrastructure only.

The warm-start network of orthoroute_b200/warm.py restated in plain PyTorch,
fp32, on the CPU (torch's own conv3d, pooling and autograd), to check the
project's CUDA forward and backward kernels.  It follows the same
architecture and weight layout:

* weights w[tap][ci][co] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1) and
  y[v] = sum_tap x[v + (dz, dy, dx)] w[tap] - a cross-correlation with zero
  padding, i.e. torch conv3d with weight[co][ci][dz+1][dy+1][dx+1];
* activations [D][H][W][C] (channels last) on the interface.

`tests/test_warm_oracle.py` pins this restatement against finite differences
in float64.
"""
from __future__ import annotations

import torch
import torch.nn.functional as Fn

LAYERS = [("e0a", True), ("e0b", True), ("e1a", True), ("e1b", True), ("e2a", True), ("e2b", True),
          ("e3a", True), ("e3b", True), ("d2", True), ("d1", True), ("d0", True), ("head", False)]


def torch_weight(w: torch.Tensor) -> torch.Tensor:
    """[27][ci][co] -> torch conv3d weight [co][ci][3][3][3]."""
    ci, co = w.shape[1], w.shape[2]
    return w.reshape(3, 3, 3, ci, co).permute(4, 3, 0, 1, 2).contiguous()


def conv(x: torch.Tensor, w: torch.Tensor, b: torch.Tensor, relu: bool) -> torch.Tensor:
    """x [1][C][D][H][W]."""
    y = Fn.conv3d(x, torch_weight(w), b, padding=1)
    return torch.relu(y) if relu else y


def forward(params: dict, x: torch.Tensor) -> torch.Tensor:
    """params: name -> (w [27][ci][co], b [co]) tensors; x: [D][H][W][16]
    channels last.  Returns the head output [D][H][W][16]."""
    h = x.permute(3, 0, 1, 2).unsqueeze(0)
    act = {}
    for lev in range(4):
        if lev > 0:
            h = Fn.avg_pool3d(act[f"e{lev - 1}b"], (1, 2, 2))
        a = conv(h, *params[f"e{lev}a"], True)
        act[f"e{lev}b"] = conv(a, *params[f"e{lev}b"], True)
    h = act["e3b"]
    for lev in (2, 1, 0):
        up = h.repeat_interleave(2, dim=3).repeat_interleave(2, dim=4)
        h = conv(up + act[f"e{lev}b"], *params[f"d{lev}"], True)
    out = conv(h, *params["head"], False)
    return out.squeeze(0).permute(1, 2, 3, 0)


def loss_fn(out: torch.Tensor, target: torch.Tensor, used: int = 2) -> torch.Tensor:
    """Mean squared error over the first `used` channels."""
    return ((out[..., :used] - target) ** 2).mean()


def grads(params: dict, x: torch.Tensor, target: torch.Tensor, dtype=torch.float32):
    """(loss, {name: (dw, db)}) by autograd."""
    p = {k: (w.detach().to(dtype).clone().requires_grad_(True), b.detach().to(dtype).clone().requires_grad_(True))
         for k, (w, b) in params.items()}
    out = forward(p, x.to(dtype))
    loss = loss_fn(out, target.to(dtype))
    loss.backward()
    return loss.detach(), {k: (w.grad, b.grad) for k, (w, b) in p.items()}
