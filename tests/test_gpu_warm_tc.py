"""The tensor-core (tcgen05.mma, TMEM accumulator) convolution of the warm
start, orsp_warm_conv3d_tc, through the C ABI: against the fp32 CPU oracle
(relative L2 error 2e-2, as the WMMA kernel's test) and against the WMMA
kernel orsp_warm_conv3d (the same bf16 products summed in another order:
1e-4 on fp32 outputs), on partial and multiple 128-voxel tiles, with and
without the ReLU mask, fp32 and bf16 outputs; and the whole network's
forward pass with either kernel."""
import numpy as np
import pytest
import torch

from oracle import warm_ref as R

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.double().flatten()
    b = b.double().flatten()
    return float((a - b).norm() / max(float(b.norm()), 1e-12))


def _bf(x):
    return x.to(torch.bfloat16).float()


def _status():
    import ctypes

    from orthoroute_b200 import _lib

    v = ctypes.c_int32(-1)
    assert _lib.load().orsp_warm_tc_status(ctypes.byref(v)) == 0
    return v.value


@pytest.mark.parametrize("cin,cout,relu,masked,W", [(16, 32, True, False, 70), (32, 32, False, True, 260),
                                                    (32, 16, True, True, 128), (32, 64, True, False, 131),
                                                    (16, 16, False, False, 9)])
def test_conv3d_tc_matches_oracle_and_wmma(cin, cout, relu, masked, W):
    from orthoroute_b200 import _lib
    from orthoroute_b200._lib import ptr

    D, H = 3, 5
    g = torch.Generator().manual_seed(cin + 3 * cout + W)
    x = _bf(torch.randn(D, H, W, cin, generator=g))
    m = _bf(torch.randn(D, H, W, cin, generator=g)) if masked else None
    w = torch.randn(27, cin, cout, generator=g) / np.sqrt(27 * cin)
    b = torch.randn(cout, generator=g) * 0.1
    wb = _bf(w)
    xm = x * (m > 0) if masked else x
    ref = R.conv(xm.permute(3, 0, 1, 2).unsqueeze(0), wb, b, relu).squeeze(0).permute(1, 2, 3, 0)
    xd = x.cuda().to(torch.bfloat16)
    md = m.cuda().to(torch.bfloat16) if masked else None
    wd = wb.cuda().to(torch.bfloat16).contiguous()
    bd = b.cuda()
    lib = _lib.load()
    y_tc = torch.full((D, H, W, cout), float("nan"), dtype=torch.float32, device="cuda")
    y_mm = torch.empty(D, H, W, cout, dtype=torch.float32, device="cuda")
    assert lib.orsp_warm_conv3d_tc(ptr(xd), ptr(md), ptr(wd), ptr(bd), None, ptr(y_tc), D, H, W, cin, cout,
                                   1 if relu else 0, 0) == 0, lib.orsp_last_error()
    assert lib.orsp_warm_conv3d(ptr(xd), ptr(md), ptr(wd), ptr(bd), None, ptr(y_mm), D, H, W, cin, cout,
                                1 if relu else 0, 0) == 0
    torch.cuda.synchronize()
    assert _status() == 0
    assert torch.isfinite(y_tc).all()
    assert _rel(y_tc.cpu(), ref) < 2e-2
    assert _rel(y_tc.cpu(), y_mm.cpu()) < 1e-4
    # bf16 output
    yb = torch.empty(D, H, W, cout, dtype=torch.bfloat16, device="cuda")
    assert lib.orsp_warm_conv3d_tc(ptr(xd), ptr(md), ptr(wd), ptr(bd), ptr(yb), None, D, H, W, cin, cout,
                                   1 if relu else 0, 0) == 0
    torch.cuda.synchronize()
    assert _rel(yb.float().cpu(), ref) < 2e-2


def test_warm_forward_tc_equals_wmma():
    from orthoroute_b200.warm import WarmNet

    net = WarmNet(C=32, seed=3)
    g = torch.Generator().manual_seed(4)
    for k in net.w:
        net.b[k].copy_(torch.randn(net.b[k].shape, generator=g) * 0.05)
    x = torch.rand(4, 48, 136, 16, generator=g).cuda().to(torch.bfloat16)
    net.conv_impl = "wmma"
    a = net.forward(x).float().cpu()
    net.conv_impl = "tc"
    b = net.forward(x).float().cpu()
    assert _status() == 0
    assert _rel(b, a) < 1e-2
