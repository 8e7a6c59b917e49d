"""The BF16 U-Net kernels (forward, backward, Adam) against a PyTorch-CPU FP64
restatement of the same network that rounds stored activations to BF16.

Single layers are checked on identical BF16 inputs against FP64 (forward
and data gradient to one BF16 rounding, weight gradient to FP32
accumulation).  The whole network is an integration check: its forward
output agrees to 2e-2 and its parameter gradients to about 6e-2 (the GPU
accumulates in FP32 and stores BF16; small differences in the forward
activations flip BF16 roundings and reach every gradient through the loss);
a wrong index or layout gives O(1) errors.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from musoc_solver_b200 import build

    build.build()
    return torch


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("H,W", [(16, 24), (32, 32)])
def test_unet_forward_backward_matches_reference(torch_cuda, H, W):
    torch = torch_cuda
    import unet_ref

    from musoc_solver_b200.unet import UNet

    net = UNet(H, W, seed=3)
    # give the biases and the head some weight so every path matters
    rng = np.random.default_rng(1)
    for name, v in net.params.items():
        v[1].copy_(torch.from_numpy(rng.normal(0, 0.05, v[1].shape).astype(np.float32)))
    net.params["head"][0].copy_(torch.from_numpy(rng.normal(0, 0.2, 32).astype(np.float32)))
    net.sync_weights()
    x = np.zeros((1, H, W, 16), np.float32)
    x[..., :3] = rng.standard_normal((1, H, W, 3))
    net.A["x"].copy_(torch.from_numpy(x.reshape(-1, 16)).to(torch.bfloat16))
    t = rng.standard_normal(H * W).astype(np.float32)
    tt = torch.from_numpy(t).cuda()
    y = net.forward().cpu().numpy()
    net.backward(tt)
    torch.cuda.synchronize()
    st = net.state()
    xr = net.A["x"].float().cpu().numpy().reshape(1, H, W, 16)
    yr, lr, gr = unet_ref.forward_backward(st, xr, t)
    assert _rel(y, yr) < 2e-2
    assert abs(float(net.loss.item()) - lr) <= 2e-2 * lr
    errs = {}
    for name, (gw, gb) in net.gw.items():
        errs[name] = _rel(gw.cpu().numpy(), gr[f"{name}.0"])
        if np.linalg.norm(gr[f"{name}.1"]) > 1e-8:
            errs[name + ".bias"] = _rel(gb.cpu().numpy(), gr[f"{name}.1"])
    print("relative gradient errors:", {k: round(v, 4) for k, v in errs.items()})
    assert max(errs.values()) < 1.2e-1, errs
    assert np.median(list(errs.values())) < 8e-2, errs


def test_unet_adam_reduces_loss(torch_cuda):
    torch = torch_cuda
    from musoc_solver_b200.unet import UNet

    H, W = 32, 48
    net = UNet(H, W, seed=4)
    rng = np.random.default_rng(2)
    x = np.zeros((H * W, 16), np.float32)
    x[:, :3] = rng.standard_normal((H * W, 3))
    net.A["x"].copy_(torch.from_numpy(x).to(torch.bfloat16))
    # a smooth target that depends on the inputs: a learnable map
    t = torch.from_numpy((0.5 * x[:, 0] - 0.3 * x[:, 1]).astype(np.float32)).cuda()
    losses = []
    for k in range(60):
        net.forward()
        net.backward(t)
        net.adam_step(lr=2e-3)
        losses.append(float(net.loss.item()))
    assert losses[-1] < 0.3 * losses[0]


def _bf(torch, a):
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16)


@pytest.mark.parametrize("cin,cout,H,W", [(16, 32, 8, 16), (64, 128, 16, 8), (256, 128, 8, 8)])
def test_conv_layer_forward_dgrad_wgrad(torch_cuda, cin, cout, H, W):
    """One 3x3 layer: forward (+bias, ReLU), masked data gradient and weight
    gradient against torch FP64 on the same BF16 values."""
    torch = torch_cuda
    import ctypes as C

    import torch.nn.functional as F

    from musoc_solver_b200.unet import lib

    L = lib()
    rng = np.random.default_rng(cin + cout)
    x = _bf(torch, rng.standard_normal((H * W, cin)))
    w = _bf(torch, rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (9, cin, cout)))
    b = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32))
    dy = _bf(torch, rng.standard_normal((H * W, cout)))
    xd, wd, bd, dyd = x.cuda(), w.cuda(), b.cuda(), dy.cuda()
    y = torch.zeros((H * W, cout), dtype=torch.bfloat16, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    assert L.sevp_nn_conv3x3(p(xd), cin, 0, cin, p(wd), p(bd), p(y), cout, 0, cout, 1, H, W, 1, None,
                             0, 0, 0, None) == 0
    # reference in FP64 from the same BF16 values
    xr = x.double().reshape(1, H, W, cin).permute(0, 3, 1, 2)
    wr = w.double().reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
    yr = F.relu(F.conv2d(xr, wr, bias=b.double(), padding=1)).permute(0, 2, 3, 1).reshape(H * W, cout)
    yg = y.double().cpu()
    assert (torch.norm(yg - yr) / torch.norm(yr)).item() < 4e-3
    # masked data gradient: dX = conv^T(dY * (y > 0))
    wt = torch.zeros((9, cout, cin), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_weight_transpose(p(wd), p(wt), cin, cout, None) == 0
    dx = torch.zeros((H * W, cin), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_conv3x3(p(dyd), cout, 0, cout, p(wt), None, p(dx), cin, 0, cin, 1, H, W, 0, p(y),
                             cout, 0, 1, None) == 0
    gm = (dy.double() * (yg > 0)).reshape(1, H, W, cout).permute(0, 3, 1, 2)
    dxr = torch.nn.grad.conv2d_input((1, cin, H, W), wr, gm, padding=1)
    dxr = dxr.permute(0, 2, 3, 1).reshape(H * W, cin)
    assert (torch.norm(dx.double().cpu() - dxr) / torch.norm(dxr)).item() < 4e-3
    # weight and bias gradients (FP32 accumulation)
    dw = torch.zeros((9, cin, cout), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    assert L.sevp_nn_conv3x3_wgrad(p(xd), cin, 0, cin, p(dyd), cout, 0, cout, p(y), cout, 0, p(dw),
                                   p(db), 1, H, W, None) == 0
    dwr = torch.nn.grad.conv2d_weight(xr, (cout, cin, 3, 3), gm, padding=1)  # co, ci, ky, kx
    dwr = dwr.permute(2, 3, 1, 0).reshape(9, cin, cout)
    assert (torch.norm(dw.double().cpu() - dwr) / torch.norm(dwr)).item() < 1e-5
    dbr = gm.sum(dim=(0, 2, 3))
    assert (torch.norm(db.double().cpu() - dbr) / torch.norm(dbr)).item() < 1e-5


@pytest.mark.parametrize("cin,cout,H,W,in_ld,in_off,out_ld,out_off",
                         [(16, 32, 8, 16, 16, 0, 32, 0), (32, 32, 24, 40, 32, 0, 64, 32),
                          (32, 64, 5, 31, 32, 0, 64, 0), (64, 64, 12, 20, 128, 64, 64, 0),
                          (64, 128, 16, 8, 64, 0, 256, 128), (128, 256, 8, 8, 128, 0, 256, 0),
                          (256, 256, 6, 10, 256, 0, 256, 0), (256, 128, 8, 8, 256, 0, 128, 0)])
def test_conv_tcgen05_forward(torch_cuda, cin, cout, H, W, in_ld, in_off, out_ld, out_off):
    """The tcgen05 forward conv (K-major weights, channel offsets of
    concatenated buffers, ragged last tile) against torch FP64 on the same
    BF16 values, and against the warp-MMA kernel; no timeout recorded."""
    torch = torch_cuda
    import ctypes as C

    import torch.nn.functional as F

    from musoc_solver_b200.unet import lib

    L = lib()
    rng = np.random.default_rng(cin * 7 + cout)
    P = H * W
    x = _bf(torch, rng.standard_normal((P, in_ld)))
    w = _bf(torch, rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (9, cin, cout)))
    b = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32))
    xd, wd, bd = x.cuda(), w.cuda(), b.cuda()
    wk = wd.permute(0, 2, 1).contiguous()
    y = torch.full((P, out_ld), 7.0, dtype=torch.bfloat16, device="cuda")
    y2 = torch.zeros((P, cout), dtype=torch.bfloat16, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    assert L.sevp_nn_conv3x3_tc(p(xd), in_ld, in_off, cin, p(wk), p(bd), p(y), out_ld, out_off, cout,
                                1, H, W, 1, None) == 0
    assert L.sevp_nn_conv3x3(p(xd), in_ld, in_off, cin, p(wd), p(bd), p(y2), cout, 0, cout, 1, H, W,
                             1, None, 0, 0, 0, None) == 0
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    xr = x[:, in_off:in_off + cin].double().reshape(1, H, W, cin).permute(0, 3, 1, 2)
    wr = w.double().reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
    yr = F.relu(F.conv2d(xr, wr, bias=b.double(), padding=1)).permute(0, 2, 3, 1).reshape(P, cout)
    yg = y.double().cpu()
    assert (torch.norm(yg[:, out_off:out_off + cout] - yr) / torch.norm(yr)).item() < 4e-3
    # channels outside [out_off, out_off + cout) are untouched
    rest = torch.cat([yg[:, :out_off], yg[:, out_off + cout:]], dim=1)
    assert bool((rest == 7.0).all())
    # same FP32 sums, rounded to BF16: at most one BF16 step apart
    d = (yg[:, out_off:out_off + cout] - y2.double().cpu()).abs()
    assert (d <= 2 ** -7 * yr.abs().clamp(min=1e-3) + 1e-6).all()


@pytest.mark.parametrize("cin,cout,B,H,W,in_ld,in_off,out_ld,out_off",
                         [(16, 32, 1, 7, 200, 16, 0, 32, 0), (32, 32, 2, 5, 129, 64, 32, 64, 0),
                          (32, 64, 1, 4, 100, 32, 0, 128, 64),
                          (64, 32, 1, 9, 150, 64, 0, 64, 32), (64, 64, 2, 5, 40, 128, 64, 64, 0),
                          (128, 64, 1, 6, 256, 128, 0, 128, 64), (256, 128, 1, 4, 130, 256, 0, 128, 0),
                          (128, 256, 1, 3, 20, 128, 0, 256, 0), (256, 256, 1, 2, 300, 256, 0, 256, 0)])
def test_conv_tma_forward(torch_cuda, cin, cout, B, H, W, in_ld, in_off, out_ld, out_off):
    """The TMA-fed tcgen05 conv (row tiles, ragged row ends, rows shorter than
    a tile, two images, channel offsets) equals the cp.async tcgen05 conv
    (the same MMA order) and matches torch FP64 on the same BF16 values."""
    torch = torch_cuda
    import ctypes as C

    import torch.nn.functional as F

    from musoc_solver_b200.unet import lib

    L = lib()
    rng = np.random.default_rng(cin * 13 + cout + W)
    P = B * H * W
    x = _bf(torch, rng.standard_normal((P, in_ld)))
    w = _bf(torch, rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (9, cin, cout)))
    b = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32))
    xd, bd = x.cuda(), b.cuda()
    wk = w.cuda().permute(0, 2, 1).contiguous()
    y1 = torch.full((P, out_ld), 5.0, dtype=torch.bfloat16, device="cuda")
    y2 = torch.full((P, out_ld), 5.0, dtype=torch.bfloat16, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    assert L.sevp_nn_conv3x3_tma(p(xd), in_ld, in_off, cin, p(wk), p(bd), p(y1), out_ld, out_off, cout,
                                 B, H, W, 1, None) == 0
    assert L.sevp_nn_conv3x3_tc(p(xd), in_ld, in_off, cin, p(wk), p(bd), p(y2), out_ld, out_off, cout,
                                B, H, W, 1, None) == 0
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    assert torch.equal(y1, y2)
    xr = x[:, in_off:in_off + cin].double().reshape(B, H, W, cin).permute(0, 3, 1, 2)
    wr = w.double().reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
    yr = F.relu(F.conv2d(xr, wr, bias=b.double(), padding=1)).permute(0, 2, 3, 1).reshape(P, cout)
    yg = y1.double().cpu()
    assert (torch.norm(yg[:, out_off:out_off + cout] - yr) / torch.norm(yr)).item() < 4e-3
    rest = torch.cat([yg[:, :out_off], yg[:, out_off + cout:]], dim=1)
    assert bool((rest == 5.0).all())


def test_conv_tcgen05_rejects_bad_shapes(torch_cuda):
    torch = torch_cuda
    import ctypes as C

    from musoc_solver_b200.unet import lib

    L = lib()
    t = torch.zeros(4096, dtype=torch.bfloat16, device="cuda")
    f = torch.zeros(256, dtype=torch.float32, device="cuda")
    p = lambda a: C.c_void_p(a.data_ptr())
    # cin not in {16..256 powers of two}, cout above 256, misaligned offset
    assert L.sevp_nn_conv3x3_tc(p(t), 48, 0, 48, p(t), p(f), p(t), 32, 0, 32, 1, 2, 2, 1, None) == 5
    assert L.sevp_nn_conv3x3_tc(p(t), 16, 0, 16, p(t), p(f), p(t), 512, 0, 512, 1, 2, 2, 1, None) == 5
    assert L.sevp_nn_conv3x3_tc(p(t), 32, 4, 16, p(t), p(f), p(t), 32, 0, 32, 1, 2, 2, 1, None) == 5


@pytest.mark.parametrize("Cc", [16, 4])
def test_pool_upsample_exact(torch_cuda, Cc):
    """2x2 average pooling and nearest upsampling, exactly (8-channel
    vector kernels for Cc = 16, one-element kernels for Cc = 4)."""
    torch = torch_cuda
    import ctypes as C

    import torch.nn.functional as F

    from musoc_solver_b200.unet import lib

    L = lib()
    H, W = 8, 12
    rng = np.random.default_rng(9)
    x = _bf(torch, rng.standard_normal((H * W, Cc))).cuda()
    p = lambda t: C.c_void_p(t.data_ptr())
    pooled = torch.zeros((H * W // 4, Cc), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_pool(p(x), Cc, 0, p(pooled), Cc, 0, Cc, 1, H, W, 0, 0, None) == 0
    xr = x.double().cpu().reshape(1, H, W, Cc).permute(0, 3, 1, 2)
    pr = F.avg_pool2d(xr, 2).permute(0, 2, 3, 1).reshape(-1, Cc).to(torch.bfloat16)
    assert torch.equal(pooled.cpu(), pr)
    up = torch.zeros((H * W, Cc), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_upsample(p(pooled), Cc, 0, p(up), Cc, 0, Cc, 1, H, W, 0, None) == 0
    ur = F.interpolate(pooled.double().cpu().reshape(1, H // 2, W // 2, Cc).permute(0, 3, 1, 2),
                       scale_factor=2, mode="nearest").permute(0, 2, 3, 1).reshape(-1, Cc)
    assert torch.equal(up.double().cpu(), ur)


def test_tma_conv_wait_timeout_is_reported_and_recovers(torch_cuda):
    """The bounded mbarrier waits of the TMA convolution: with the wait limit
    set to zero polls every tile gives up at its first wait, records
    SEVP_TIMEOUT (read by sevp_nn_tc_status), skips its stores and returns
    after draining the copies it issued; with the default limit restored the
    same call computes the convolution again and reports no error."""
    import ctypes as C

    import torch

    from musoc_solver_b200.unet import lib as nnlib

    L = nnlib()
    H, W, cin, cout = 64, 128, 64, 32
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(H * W, cin, device="cuda", generator=g).to(torch.bfloat16)
    wk = (torch.randn(9, cout, cin, device="cuda", generator=g) / 30).to(torch.bfloat16)
    bias = torch.zeros(cout, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0
    try:
        assert L.sevp_nn_tc_set_wait_limit(0) == 0
        y = torch.full((H * W, cout), 7.0, dtype=torch.bfloat16, device="cuda")
        assert L.sevp_nn_conv3x3_tma(ptr(x), cin, 0, cin, ptr(wk), ptr(bias), ptr(y), cout, 0,
                                     cout, 1, H, W, 1, None) == 0
        assert L.sevp_nn_tc_status(C.byref(code)) == 0
        assert code.value == 4  # SEVP_TIMEOUT
        assert bool((y == 7.0).all())  # no tile stored a result
    finally:
        assert L.sevp_nn_tc_set_wait_limit(0xFFFFFFFF) == 0
    y = torch.zeros((H * W, cout), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_conv3x3_tma(ptr(x), cin, 0, cin, ptr(wk), ptr(bias), ptr(y), cout, 0, cout, 1,
                                 H, W, 1, None) == 0
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    y2 = torch.zeros_like(y)
    assert L.sevp_nn_conv3x3_tc(ptr(x), cin, 0, cin, ptr(wk), ptr(bias), ptr(y2), cout, 0, cout, 1,
                                H, W, 1, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(y, y2)


@pytest.mark.parametrize("cin,cout,B,H,W,dy_ld,dy_off,dx_ld,dx_off",
                         [(32, 32, 1, 8, 16, 32, 0, 64, 32), (64, 32, 1, 9, 150, 64, 32, 64, 0),
                          (32, 64, 2, 5, 40, 128, 64, 32, 0), (128, 128, 1, 6, 130, 256, 128, 256, 0),
                          (256, 128, 1, 4, 20, 128, 0, 256, 0), (128, 256, 1, 3, 24, 256, 0, 128, 0)])
def test_conv_dgrad_tcgen05(torch_cuda, cin, cout, B, H, W, dy_ld, dy_off, dx_ld, dx_off):
    """The data gradient on the tcgen05 tensor cores (masked output gradient
    packed, then a TMA forward conv with the tap-mirrored weights) against
    torch FP64 on the same BF16 values, to one BF16 rounding, and within one
    BF16 step of the warp-MMA data gradient."""
    torch = torch_cuda
    import ctypes as C

    from musoc_solver_b200.unet import lib

    L = lib()
    rng = np.random.default_rng(cin * 5 + cout + W)
    P = B * H * W
    w = _bf(torch, rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (9, cin, cout)))
    dy = _bf(torch, rng.standard_normal((P, dy_ld)))
    mask = _bf(torch, rng.standard_normal((P, cout)))  # forward output: ReLU passes where > 0
    wd, dyd, md = w.cuda(), dy.cuda(), mask.cuda()
    p = lambda t: C.c_void_p(t.data_ptr())
    wm = torch.zeros_like(wd)
    assert L.sevp_nn_weight_mirror(p(wd), p(wm), cin, cout, None) == 0
    scratch = torch.zeros(P * cout, dtype=torch.bfloat16, device="cuda")
    dx = torch.full((P, dx_ld), 7.0, dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_conv3x3_dgrad_tc(p(dyd), dy_ld, dy_off, cout, p(md), cout, 0, p(wm), p(scratch),
                                      p(dx), dx_ld, dx_off, cin, B, H, W, None) == 0
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    wr = w.double().reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
    gm = (dy[:, dy_off:dy_off + cout].double() * (mask.double() > 0))
    gm = gm.reshape(B, H, W, cout).permute(0, 3, 1, 2)
    dxr = torch.nn.grad.conv2d_input((B, cin, H, W), wr, gm, padding=1)
    dxr = dxr.permute(0, 2, 3, 1).reshape(P, cin)
    dg = dx.double().cpu()
    assert (torch.norm(dg[:, dx_off:dx_off + cin] - dxr) / torch.norm(dxr)).item() < 4e-3
    rest = torch.cat([dg[:, :dx_off], dg[:, dx_off + cin:]], dim=1)
    assert bool((rest == 7.0).all())
    # the warp-MMA data gradient of the same values
    wt = torch.zeros((9, cout, cin), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_weight_transpose(p(wd), p(wt), cin, cout, None) == 0
    dx2 = torch.zeros((P, cin), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_conv3x3(p(dyd), dy_ld, dy_off, cout, p(wt), None, p(dx2), cin, 0, cin, B, H, W,
                             0, p(md), cout, 0, 1, None) == 0
    d = (dg[:, dx_off:dx_off + cin] - dx2.double().cpu()).abs()
    assert (d <= 2 ** -7 * dxr.abs().clamp(min=1e-3) + 1e-6).all()


def test_unet_layers_through_the_network(torch_cuda):
    """Every convolution of a whole forward and backward pass, checked where
    it runs: each layer's output, weight and bias gradients and data
    gradient against torch FP64 on the BF16 values the network actually fed
    it (its wiring: sources, channel offsets, masks, concatenations).
    Forward outputs and data gradients to one BF16 rounding, weight and bias
    gradients to FP32 accumulation."""
    torch = torch_cuda
    import torch.nn.functional as F

    from musoc_solver_b200.unet import CONVS, UNet

    H, W = 32, 48
    net = UNet(H, W, seed=5)
    rng = np.random.default_rng(6)
    for name, v in net.params.items():
        v[1].copy_(torch.from_numpy(rng.normal(0, 0.05, v[1].shape).astype(np.float32)))
    net.params["head"][0].copy_(torch.from_numpy(rng.normal(0, 0.2, 32).astype(np.float32)))
    net.sync_weights()
    x = np.zeros((H * W, 16), np.float32)
    x[:, :3] = rng.standard_normal((H * W, 3))
    net.A["x"].copy_(torch.from_numpy(x).to(torch.bfloat16))
    t = torch.from_numpy(rng.standard_normal(H * W).astype(np.float32)).cuda()
    # one training step first: the checked pass runs on updated weights (and
    # their derived copies, which the data gradient reads)
    net.forward()
    net.backward(t)
    net.adam_step(lr=1e-2)
    torch.cuda.synchronize()
    dims = {n: (ci, co) for n, ci, co in CONVS}
    errs = {}

    def region(tns, off, ld, c, lvl):
        h, w = H >> lvl, W >> lvl
        a = tns.reshape(-1, ld)[:, off:off + c].double().cpu()
        return a.reshape(1, h, w, c).permute(0, 3, 1, 2)

    def wref(name):
        ci, co = dims[name]
        return net.w16[name].double().cpu().reshape(3, 3, ci, co).permute(3, 2, 0, 1)

    conv_f, conv_b = net._conv, net._conv_bwd

    def rel(a, b):
        return (torch.norm(a - b) / max(torch.norm(b).item(), 1e-30)).item()

    def checked_conv(name, src, src_off, src_ld, dst, dst_off, dst_ld, lvl):
        ci, co = dims[name]
        xr = region(src, src_off, src_ld, ci, lvl)
        conv_f(name, src, src_off, src_ld, dst, dst_off, dst_ld, lvl)
        torch.cuda.synchronize()
        yr = F.relu(F.conv2d(xr, wref(name), bias=net.params[name][1].double().cpu(), padding=1))
        errs[name + ".fwd"] = rel(region(dst, dst_off, dst_ld, co, lvl), yr)

    def checked_bwd(name, src, src_off, src_ld, gout, gout_off, gout_ld, out, out_off, out_ld,
                    dsrc, dsrc_off, dsrc_ld, lvl):
        ci, co = dims[name]
        xr = region(src, src_off, src_ld, ci, lvl)
        gm = region(gout, gout_off, gout_ld, co, lvl) * (region(out, out_off, out_ld, co, lvl) > 0)
        conv_b(name, src, src_off, src_ld, gout, gout_off, gout_ld, out, out_off, out_ld, dsrc,
               dsrc_off, dsrc_ld, lvl)
        torch.cuda.synchronize()
        dwr = torch.nn.grad.conv2d_weight(xr, (co, ci, 3, 3), gm, padding=1)
        dwr = dwr.permute(2, 3, 1, 0).reshape(9, ci, co)
        gw, gb = net.gw[name]
        errs[name + ".wgrad"] = rel(gw.double().cpu(), dwr)
        errs[name + ".bgrad"] = rel(gb.double().cpu(), gm.sum(dim=(0, 2, 3)))
        if dsrc is not None:
            dxr = torch.nn.grad.conv2d_input(xr.shape, wref(name), gm, padding=1)
            errs[name + ".dgrad"] = rel(region(dsrc, dsrc_off, dsrc_ld, ci, lvl), dxr)

    net._conv, net._conv_bwd = checked_conv, checked_bwd
    net.forward()
    net.backward(t)
    torch.cuda.synchronize()
    kinds = {k.rsplit(".", 1)[1] for k in errs}
    assert kinds == {"fwd", "wgrad", "bgrad", "dgrad"}
    assert sum(k.endswith(".fwd") for k in errs) == len(CONVS)
    assert sum(k.endswith(".wgrad") for k in errs) == len(CONVS)
    assert sum(k.endswith(".dgrad") for k in errs) == len(CONVS) - 1
    bad = {k: v for k, v in errs.items()
           if v >= (4e-3 if k.endswith((".fwd", ".dgrad")) else 1e-5)}
    assert not bad, bad


@pytest.mark.parametrize("cin,cout,B,H,W,x_ld,x_off",
                         [(16, 32, 1, 8, 16, 16, 0), (32, 64, 1, 9, 150, 64, 32),
                          (64, 32, 2, 5, 40, 128, 64), (128, 128, 1, 6, 130, 256, 128),
                          (256, 128, 1, 4, 20, 256, 0), (128, 256, 1, 3, 24, 128, 0)])
def test_conv_wgrad_tcgen05(torch_cuda, cin, cout, B, H, W, x_ld, x_off):
    """The weight gradient on the tcgen05 tensor cores (pixel-contraction
    GEMM per tap, split over CTAs, FP32 atomics) against torch FP64 on the
    same BF16 values, to FP32 accumulation; the whole backward call
    (packing, weight, bias and data gradients) against the separate pieces."""
    torch = torch_cuda
    import ctypes as C

    import torch.nn.functional as F  # noqa: F401

    from musoc_solver_b200.unet import lib

    L = lib()
    rng = np.random.default_rng(cin * 3 + cout + W)
    P = B * H * W
    x = _bf(torch, rng.standard_normal((P, x_ld)))
    g = _bf(torch, rng.standard_normal((P, cout)))
    xd, gd = x.cuda(), g.cuda()
    p = lambda t: C.c_void_p(t.data_ptr())
    dw = torch.zeros((9, cin, cout), dtype=torch.float32, device="cuda")
    assert L.sevp_nn_conv3x3_wgrad_tc(p(xd), x_ld, x_off, cin, p(gd), cout, p(dw), B, H, W,
                                      None) == 0
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    xr = x[:, x_off:x_off + cin].double().reshape(B, H, W, cin).permute(0, 3, 1, 2)
    gr = g.double().reshape(B, H, W, cout).permute(0, 3, 1, 2)
    dwr = torch.nn.grad.conv2d_weight(xr, (cout, cin, 3, 3), gr, padding=1)
    dwr = dwr.permute(2, 3, 1, 0).reshape(9, cin, cout)
    assert (torch.norm(dw.double().cpu() - dwr) / torch.norm(dwr)).item() < 1e-5
    # accumulates: a second call doubles it
    assert L.sevp_nn_conv3x3_wgrad_tc(p(xd), x_ld, x_off, cin, p(gd), cout, p(dw), B, H, W,
                                      None) == 0
    assert (torch.norm(dw.double().cpu() - 2 * dwr) / torch.norm(2 * dwr)).item() < 1e-5
    # the combined backward with a ReLU mask
    mask = _bf(torch, rng.standard_normal((P, cout))).cuda()
    w = _bf(torch, rng.normal(0, (2.0 / (9 * cin)) ** 0.5, (9, cin, cout))).cuda()
    wm = torch.zeros_like(w)
    assert L.sevp_nn_weight_mirror(p(w), p(wm), cin, cout, None) == 0
    scratch = torch.zeros(P * cout, dtype=torch.bfloat16, device="cuda")
    dw2 = torch.zeros_like(dw)
    db2 = torch.zeros(cout, dtype=torch.float32, device="cuda")
    dx2 = torch.zeros((P, cin), dtype=torch.bfloat16, device="cuda")
    assert L.sevp_nn_conv3x3_backward_tc(p(xd), x_ld, x_off, cin, p(gd), cout, 0, cout, p(mask),
                                         cout, 0, p(wm), p(scratch), p(dw2), p(db2), p(dx2), cin, 0,
                                         B, H, W, None) == 0
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    gm = (g.double() * (mask.double().cpu() > 0)).reshape(B, H, W, cout).permute(0, 3, 1, 2)
    dwm = torch.nn.grad.conv2d_weight(xr, (cout, cin, 3, 3), gm, padding=1)
    dwm = dwm.permute(2, 3, 1, 0).reshape(9, cin, cout)
    assert (torch.norm(dw2.double().cpu() - dwm) / torch.norm(dwm)).item() < 1e-5
    dbm = gm.sum(dim=(0, 2, 3))
    assert (torch.norm(db2.double().cpu() - dbm) / torch.norm(dbm)).item() < 1e-5
    wr = w.double().cpu().reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
    dxr = torch.nn.grad.conv2d_input((B, cin, H, W), wr, gm, padding=1).permute(0, 2, 3, 1)
    dxr = dxr.reshape(P, cin)
    assert (torch.norm(dx2.double().cpu() - dxr) / torch.norm(dxr)).item() < 4e-3


def test_conv_wgrad_tcgen05_bounded_wait(torch_cuda):
    """The weight-gradient kernel's bounded waits: with the poll limit at 0
    every CTA gives up at its first wait for a stage (each has five steps of
    64 pixels here), drains the MMAs it issued, adds nothing to dw and
    records SEVP_TIMEOUT; with the limit restored the same call is exact."""
    torch = torch_cuda
    import ctypes as C

    from musoc_solver_b200.unet import lib

    L = lib()
    cin, cout, H, W = 32, 32, 64, 160
    rng = np.random.default_rng(9)
    x = _bf(torch, rng.standard_normal((H * W, cin))).cuda()
    g = _bf(torch, rng.standard_normal((H * W, cout))).cuda()
    dw = torch.zeros((9, cin, cout), dtype=torch.float32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0
    try:
        assert L.sevp_nn_tc_set_wait_limit(0) == 0
        assert L.sevp_nn_conv3x3_wgrad_tc(p(x), cin, 0, cin, p(g), cout, p(dw), 1, H, W, None) == 0
        assert L.sevp_nn_tc_status(C.byref(code)) == 0
        assert code.value == 4  # SEVP_TIMEOUT
        assert bool((dw == 0).all())
    finally:
        assert L.sevp_nn_tc_set_wait_limit(0xFFFFFFFF) == 0
    assert L.sevp_nn_conv3x3_wgrad_tc(p(x), cin, 0, cin, p(g), cout, p(dw), 1, H, W, None) == 0
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    xr = x.double().cpu().reshape(1, H, W, cin).permute(0, 3, 1, 2)
    gr = g.double().cpu().reshape(1, H, W, cout).permute(0, 3, 1, 2)
    dwr = torch.nn.grad.conv2d_weight(xr, (cout, cin, 3, 3), gr, padding=1)
    dwr = dwr.permute(2, 3, 1, 0).reshape(9, cin, cout)
    assert (torch.norm(dw.double().cpu() - dwr) / torch.norm(dwr)).item() < 1e-5
