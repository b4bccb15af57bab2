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


@pytest.mark.parametrize("cin,cout,relu,masked,W,D,H", [(16, 32, True, False, 70, 3, 5), (32, 32, False, True, 260, 3, 5),
                                                        (32, 16, True, True, 128, 3, 5), (32, 64, True, False, 131, 3, 5),
                                                        (16, 16, False, False, 9, 3, 5),
                                                        (32, 32, True, True, 200, 6, 40),
                                                        (32, 64, False, False, 131, 4, 60)])
@pytest.mark.parametrize("kernel", ["warp-specialised", "stage-barrier"])
def test_conv3d_tc_matches_oracle_and_wmma(cin, cout, relu, masked, W, D, H, kernel, monkeypatch):
    """The tensor-core convolution against the fp32 oracle and the WMMA
    kernel: partial and several tiles per row, with and without the ReLU
    mask, bf16 and fp32 outputs; the last two shapes give every CTA about
    three tiles (480 tiles on 148 CTAs), so the epilogue of one tile runs
    beside the next tile's MMAs in both accumulators.  Both kernels: the
    warp-specialised one (producer warps, an MMA warp, mbarrier handoffs) and
    the one with a block barrier per stage (ORSP_WARM_TC_WS=0)."""
    from orthoroute_b200 import _lib
    from orthoroute_b200._lib import ptr

    monkeypatch.setenv("ORSP_WARM_TC_WS", "0" if kernel == "stage-barrier" else "1")

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


@pytest.mark.parametrize("cin,cout,masked,W", [(16, 32, True, 70), (32, 32, False, 41), (32, 16, True, 96)])
def test_wgrad_tc_matches_wmma(cin, cout, masked, W):
    """orsp_warm_wgrad_tc against orsp_warm_wgrad: the same bf16 products
    summed in fp32 in another order (relative L2 error 1e-4), weights and
    biases, accumulated into existing values."""
    from orthoroute_b200 import _lib
    from orthoroute_b200._lib import ptr

    D, H = 3, 6
    g = torch.Generator().manual_seed(11 + cin + cout + W)
    x = torch.randn(D, H, W, cin, generator=g).cuda().to(torch.bfloat16)
    dy = torch.randn(D, H, W, cout, generator=g).cuda().to(torch.bfloat16)
    yo = torch.randn(D, H, W, cout, generator=g).cuda().to(torch.bfloat16) if masked else None
    lib = _lib.load()
    base_w = torch.randn(27 * cin * cout, generator=g).cuda()
    base_b = torch.randn(cout, generator=g).cuda()
    dw_tc, db_tc = base_w.clone(), base_b.clone()
    dw_mm, db_mm = base_w.clone(), base_b.clone()
    assert lib.orsp_warm_wgrad_tc(ptr(x), ptr(dy), ptr(yo), ptr(dw_tc), ptr(db_tc), D, H, W, cin, cout, 0) == 0, \
        lib.orsp_last_error()
    assert lib.orsp_warm_wgrad(ptr(x), ptr(dy), ptr(yo), ptr(dw_mm), ptr(db_mm), D, H, W, cin, cout, 0) == 0
    torch.cuda.synchronize()
    assert _status() == 0
    assert _rel((dw_tc - base_w).cpu(), (dw_mm - base_w).cpu()) < 1e-4
    assert _rel((db_tc - base_b).cpu(), (db_mm - base_b).cpu()) < 1e-4


def test_warm_gradients_tc_match_oracle():
    """A forward and backward pass of the whole network on the tensor-core
    kernels against the fp32 oracle's gradients (1e-1, as the WMMA path)."""
    from orthoroute_b200.warm import WarmNet

    net = WarmNet(C=32, seed=3)
    net.conv_impl = "tc"
    g = torch.Generator().manual_seed(4)
    for k in net.w:
        net.b[k].copy_(torch.randn(net.b[k].shape, generator=g) * 0.05)
    D, H, W = 3, 32, 40
    x = _bf(torch.rand(D, H, W, 16, generator=g))
    t = torch.rand(D, H, W, 2, generator=g)
    params = {k: (_bf(net.w[k].cpu()), net.b[k].cpu()) for k in net.w}
    out, act = net.forward(x.cuda().to(torch.bfloat16), keep=True)
    loss, dout = net.loss_grad(out, t.cuda().contiguous())
    net.backward(act, dout)
    torch.cuda.synchronize()
    assert _status() == 0
    ref_loss, ref_g = R.grads(params, x, t)
    assert abs(float(loss) - float(ref_loss)) < 5e-2 * float(ref_loss)
    err = {k: (round(_rel(net.gw[k].cpu(), ref_g[k][0]), 4), round(_rel(net.gb[k].cpu(), ref_g[k][1]), 4))
           for k in net.w}
    assert max(max(v) for v in err.values()) < 1e-1, err
