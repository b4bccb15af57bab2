"""The warm-start network's CUDA kernels (orsp_warm.cu, through the C ABI)
against the fp32 CPU oracle (oracle/warm_ref.py).  Activations are bf16 with
fp32 accumulation, so results are compared by relative L2 error: 2e-2 for one
convolution, 5e-2 for the 12-layer forward pass, 1e-1 for weight and bias
gradients (bf16 gradients through 12 layers)."""
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


@pytest.mark.parametrize("cin,cout,relu,masked", [(16, 32, True, False), (32, 32, False, True), (32, 16, True, True)])
def test_conv3d_kernel_matches_oracle(cin, cout, relu, masked):
    from orthoroute_b200 import _lib
    from orthoroute_b200._lib import ptr

    D, H, W = 3, 5, 70  # W not a multiple of the 64-voxel tile
    g = torch.Generator().manual_seed(cin + cout)
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
    y = torch.empty(D, H, W, cout, dtype=torch.float32, device="cuda")
    st = _lib.load().orsp_warm_conv3d(ptr(xd), ptr(md), ptr(wd), ptr(bd), None, ptr(y), D, H, W, cin, cout,
                                      1 if relu else 0, 0)
    assert st == 0
    assert _rel(y.cpu(), ref) < 2e-2


def _net_and_data(seed=0):
    from orthoroute_b200.warm import WarmNet

    net = WarmNet(C=32, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    for k in net.w:  # non-zero biases exercise the bias paths
        net.b[k].copy_(torch.randn(net.b[k].shape, generator=g) * 0.05)
    D, H, W = 3, 32, 40  # the bottleneck level keeps 3 x 4 x 5 voxels
    x = _bf(torch.rand(D, H, W, 16, generator=g))
    t = torch.rand(D, H, W, 2, generator=g)
    params = {k: (_bf(net.w[k].cpu()), net.b[k].cpu()) for k in net.w}
    return net, params, x, t


def test_warm_forward_matches_oracle():
    net, params, x, _ = _net_and_data()
    out = net.forward(x.cuda().to(torch.bfloat16)).cpu()
    ref = R.forward(params, x)
    assert _rel(out[..., :2], ref[..., :2]) < 5e-2
    assert _rel(out, ref) < 5e-2


def test_warm_gradients_match_oracle():
    net, params, x, t = _net_and_data(seed=3)
    out, act = net.forward(x.cuda().to(torch.bfloat16), keep=True)
    loss, dout = net.loss_grad(out, t.cuda().contiguous())
    net.backward(act, dout)
    torch.cuda.synchronize()
    ref_loss, ref_g = R.grads(params, x, t)
    assert abs(float(loss) - float(ref_loss)) < 5e-2 * float(ref_loss)
    err = {k: (round(_rel(net.gw[k].cpu(), ref_g[k][0]), 4), round(_rel(net.gb[k].cpu(), ref_g[k][1]), 4))
           for k in net.w}
    assert max(max(v) for v in err.values()) < 1e-1, err


def test_warm_training_lowers_loss():
    net, _, x, t = _net_and_data(seed=5)
    xd, td = x.cuda().to(torch.bfloat16), t.cuda().contiguous()
    losses = []
    for _ in range(60):
        out, act = net.forward(xd, keep=True)
        loss, dout = net.loss_grad(out, td)
        net.backward(act, dout)
        net.step(lr=3e-3)
        losses.append(float(loss))
    assert losses[-1] < 0.5 * losses[0]


def test_shipped_warm_start_gains_over_zero_history():
    """The shipped network (orthoroute_b200/data/warm_history.npz, trained on
    seeds 2000+) on an unseen 300x300x18 board at the backplane's net density:
    starting from its predicted history, PathFinder reaches zero overuse with
    fewer searches than from zero history, at wirelength within 2 %."""
    from orthoroute_b200.lattice import board_footprints
    from orthoroute_b200.negotiate import PathFinder
    from orthoroute_b200.warm import load_pretrained, warm_history
    from orthoroute_b200.warm_train import route_config

    b = board_footprints(300, 300, 18, 2000, None, seed=77)
    pf = PathFinder(b.lattice, config=route_config(60))
    r0 = pf.route(b.src, b.dst, mode="batched")
    net, scale = load_pretrained()
    rw = pf.route(b.src, b.dst, mode="batched", history_init=warm_history(net, b.lattice, b.src, b.dst, scale))
    s0 = sum(s.nets_searched for s in r0.iterations)
    sw = sum(s.nets_searched for s in rw.iterations)
    print(f"zero history: {len(r0.iterations)} iterations, {s0} searches; warm: {len(rw.iterations)} iterations, "
          f"{sw} searches; wirelength {r0.wirelength} -> {rw.wirelength}")
    assert r0.converged and rw.converged
    assert sw < s0
    assert abs(rw.wirelength - r0.wirelength) <= 0.02 * r0.wirelength


def test_warm_history_device_matches_host():
    """warm_history_device (features assembled, run and mapped to edges on
    the device) gives warm_history's per-edge history: the same network
    outputs, the same float64 expm1 and scale up to the last bit of the
    device's expm1, so at most one float32 ulp apart, on a board whose H and W
    are not multiples of 8."""
    from orthoroute_b200.lattice import board_footprints
    from orthoroute_b200.warm import load_pretrained, warm_history, warm_history_device

    from orthoroute_b200.warm import _air_counts_device, _segment_points

    b = board_footprints(203, 117, 18, 600, None, seed=5)
    lat = b.lattice
    sx, sy, _ = lat.coords(np.asarray(b.src))
    dx, dy, _ = lat.coords(np.asarray(b.dst))
    xs, ys = _segment_points(sx, sy, dx, dy)
    air = np.bincount(ys * lat.nx + xs, minlength=lat.ny * lat.nx).astype(np.float32).reshape(lat.ny, lat.nx)
    assert np.array_equal(_air_counts_device(sx, sy, dx, dy, lat.nx, lat.ny, "cuda"), air)
    net, scale = load_pretrained()
    h_host = warm_history(net, b.lattice, b.src, b.dst, scale)
    h_dev = warm_history_device(net, b.lattice, b.src, b.dst, scale)
    assert h_dev.dtype == torch.float32 and h_dev.is_cuda and h_dev.numel() == h_host.size
    hd = h_dev.cpu().numpy()
    ulp = np.abs(hd.view(np.int32).astype(np.int64) - h_host.view(np.int32).astype(np.int64))
    assert int(ulp.max()) <= 1, int(ulp.max())
    assert float(np.mean(ulp == 0)) > 0.999
