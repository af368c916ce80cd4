"""U-Net kernels of the learned preconditioner against a plain PyTorch fp32
reference on the same bf16 values.

Products are bf16 x bf16 accumulated in FP32 on both sides, so single kernels
agree to FP32 summation order (plus one bf16 rounding of stored
activations); the whole network is compared with a torch model that rounds
its activations to bf16 at the same points (straight-through in backward).
"""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

F = torch.nn.functional


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _bf(t):
    return t.to(torch.bfloat16).float()


def _relerr(a, b):
    a, b = a.detach(), b.detach()
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


def _torch_w(w, co, ci):
    """[9][co][ci] -> torch [co][ci][3][3]."""
    return w.reshape(3, 3, co, ci).permute(2, 3, 0, 1).contiguous()


def test_conv3x3_forward_data_and_weight_gradients():
    from seispie_b200 import _lib
    from seispie_b200.engine import check, ptr, stream_handle
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(3)
    n, h, w, c0, c1, co = 2, 24, 40, 32, 16, 48
    x0 = _bf(torch.randn(n, h, w, c0, device="cuda", generator=g))
    x1 = _bf(torch.randn(n, h, w, c1, device="cuda", generator=g))
    wt = _bf(torch.randn(9, co, c0 + c1, device="cuda", generator=g) * 0.1)
    b = torch.randn(co, device="cuda", generator=g)
    # bf16 copies held for as long as the queued kernels read them
    x0b, x1b, wtb = x0.bfloat16(), x1.bfloat16(), wt.bfloat16()
    out = torch.empty(n, h, w, co, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_conv3x3(ptr(x0b), c0, ptr(x1b), c1, ptr(wtb), ptr(b), co,
                               ptr(out), co, None, 0, n, h, w, 1, stream_handle(None)), "conv")
    xt = torch.cat([x0, x1], -1).permute(0, 3, 1, 2).requires_grad_(True)
    wtt = _torch_w(wt, co, c0 + c1).requires_grad_(True)
    ref = F.relu(F.conv2d(xt, wtt, b, padding=1))
    got = out.float().permute(0, 3, 1, 2)
    assert (got - ref).abs().max() <= 1e-2 * ref.abs().max()
    # data and weight gradients of a bf16 upstream gradient through the ReLU
    gy = _bf(torch.randn(n, co, h, w, device="cuda", generator=g))
    ref.backward(gy)
    gy_nhwc = gy.permute(0, 2, 3, 1).contiguous().bfloat16()
    check(lib.fwi_unet_relu_bwd(ptr(gy_nhwc), ptr(out), gy_nhwc.numel(), stream_handle(None)), "relu_bwd")
    wd = torch.empty(9 * co * (c0 + c1), dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_flip_weights(ptr(wtb), ptr(wd), co, c0 + c1, stream_handle(None)), "flip")
    gx0 = torch.empty(n, h, w, c0, dtype=torch.bfloat16, device="cuda")
    gx1 = torch.empty(n, h, w, c1, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_conv3x3(ptr(gy_nhwc), co, None, 0, ptr(wd), None, c0 + c1, ptr(gx0), c0, ptr(gx1), c1,
                               n, h, w, 0, stream_handle(None)), "dgrad")
    gx_ref = xt.grad.permute(0, 2, 3, 1)
    gx = torch.cat([gx0.float(), gx1.float()], -1)
    assert (gx - gx_ref).abs().max() <= 1e-2 * gx_ref.abs().max()
    part = torch.empty(lib.fwi_unet_wgrad_partials(co, c0 + c1, n, h, w), dtype=torch.float32, device="cuda")
    dw = torch.empty(9 * co * (c0 + c1), dtype=torch.float32, device="cuda")
    db = torch.empty(co, dtype=torch.float32, device="cuda")
    check(lib.fwi_unet_conv3x3_wgrad(ptr(gy_nhwc), co, ptr(x0b), c0, ptr(x1b), c1, n, h, w,
                                     ptr(part), ptr(dw), ptr(db), stream_handle(None)), "wgrad")
    dw_t = _torch_w(dw, co, c0 + c1)
    assert _relerr(dw_t, wtt.grad) < 1e-5
    gy_masked = gy_nhwc.float()
    assert _relerr(db, gy_masked.sum((0, 1, 2))) < 1e-5


@pytest.mark.parametrize("n,h,w,c0,c1,co,d1", [
    (2, 5, 260, 32, 16, 48, 16),    # two full strips and a 4-pixel one; concatenated input; split output
    (1, 4, 130, 16, 0, 16, 0),      # exactly one halo box wide, one chunk
    (3, 2, 64, 32, 0, 32, 0),       # narrowest image of the tcgen05 path, 2 rows: box past every edge
    (2, 1, 100, 16, 16, 32, 0),     # one row
    (1, 3, 200, 128, 0, 128, 0),    # N = 128, ring of 2 stages wrapped 4 times
    (2, 6, 140, 128, 64, 64, 0),    # N = 64, 12 chunks through a ring of 3
    (1, 7, 131, 64, 32, 32, 0),     # N = 32, 6 chunks through a ring of 4
])
def test_conv3x3_tcgen05_matches_torch_and_mma_sync(n, h, w, c0, c1, co, d1):
    """The tcgen05 kernel (images >= 130 pixels wide) against torch fp32 and
    against the mma.sync kernel on the same bf16 values."""
    from seispie_b200 import _lib
    from seispie_b200.engine import check, ptr, stream_handle
    import ctypes
    lib, st = _lib.load(), stream_handle(None)
    g = torch.Generator(device="cuda").manual_seed(11 + w)
    x0 = _bf(torch.randn(n, h, w, c0, device="cuda", generator=g)).bfloat16()
    x1 = _bf(torch.randn(n, h, w, max(c1, 16), device="cuda", generator=g)).bfloat16()
    wt = _bf(torch.randn(9, co, c0 + c1, device="cuda", generator=g) * 0.1).bfloat16()
    b = torch.randn(co, device="cuda", generator=g)
    d0 = co - d1
    outs = []
    for path in (0, 1):
        old = lib.fwi_unet_conv_path(path)
        o0 = torch.full((n, h, w, d0), float("nan"), dtype=torch.bfloat16, device="cuda")
        o1 = torch.full((n, h, w, max(d1, 16)), float("nan"), dtype=torch.bfloat16, device="cuda")
        check(lib.fwi_unet_conv3x3(ptr(x0), c0, ptr(x1) if c1 else None, c1, ptr(wt), ptr(b), co, ptr(o0), d0,
                                   ptr(o1) if d1 else None, d1, n, h, w, 1, st), "conv path %d" % path)
        lib.fwi_unet_conv_path(old)
        outs.append(torch.cat([o0.float(), o1[..., :d1].float()], -1))
    torch.cuda.synchronize()
    status = ctypes.c_int(-1)
    check(lib.fwi_device_status(ctypes.byref(status), 1), "status")
    assert status.value == 0
    xt = torch.cat([x0.float(), x1[..., :c1].float()], -1).permute(0, 3, 1, 2)
    ref = F.relu(F.conv2d(xt, _torch_w(wt.float(), co, c0 + c1), b, padding=1)).permute(0, 2, 3, 1)
    for got in outs:
        assert torch.isfinite(got).all()
        assert (got - ref).abs().max() <= 1e-2 * ref.abs().max()
    assert (outs[0] - outs[1]).abs().max() <= 1e-2 * ref.abs().max()


def test_pool_upsample_pack_head():
    from seispie_b200 import _lib
    from seispie_b200.engine import check, ptr, stream_handle
    lib, st = _lib.load(), stream_handle(None)
    g = torch.Generator(device="cuda").manual_seed(5)
    n, h, w, c = 2, 16, 24, 32
    x = _bf(torch.randn(n, h, w, c, device="cuda", generator=g)).bfloat16()
    p = torch.empty(n, h // 2, w // 2, c, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_pool2(ptr(x), ptr(p), c, n, h, w, st), "pool")
    ref = F.avg_pool2d(x.float().permute(0, 3, 1, 2), 2).permute(0, 2, 3, 1)
    assert (p.float() - ref).abs().max() <= 4e-3 * ref.abs().max()
    gp = _bf(torch.randn(n, h // 2, w // 2, c, device="cuda", generator=g)).bfloat16()
    gx = torch.zeros(n, h, w, c, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_pool2_bwd(ptr(gp), ptr(gx), c, n, h, w, 0, st), "pool_bwd")
    assert torch.equal(gx.float(), 0.25 * gp.float().repeat_interleave(2, 1).repeat_interleave(2, 2))
    u = torch.empty(n, 2 * h, 2 * w, c, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_up2(ptr(x), ptr(u), c, n, h, w, st), "up")
    assert torch.equal(u, x.repeat_interleave(2, 1).repeat_interleave(2, 2))
    gu = torch.ones(n, 2 * h, 2 * w, c, dtype=torch.bfloat16, device="cuda")
    gi = torch.empty(n, h, w, c, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_up2_bwd(ptr(gu), ptr(gi), c, n, h, w, st), "up_bwd")
    assert torch.all(gi.float() == 4.0)
    planes = torch.randn(n, 3, h, w, device="cuda", generator=g)
    xp = torch.empty(n, h, w, 16, dtype=torch.bfloat16, device="cuda")
    check(lib.fwi_unet_pack(ptr(planes), ptr(xp), n, h, w, st), "pack")
    assert torch.equal(xp[..., :3].float(), _bf(planes.permute(0, 2, 3, 1)))
    assert torch.all(xp[..., 3:] == 0)
    x16 = _bf(torch.randn(n, h, w, 16, device="cuda", generator=g)).bfloat16()
    hw = torch.randn(16, device="cuda", generator=g)
    hb = torch.randn(1, device="cuda", generator=g)
    out = torch.empty(n, h, w, device="cuda")
    check(lib.fwi_unet_head(ptr(x16), ptr(hw), ptr(hb), ptr(out), n, h, w, st), "head")
    assert _relerr(out, x16.float() @ hw + hb) < 1e-6
    gout = torch.randn(n, h, w, device="cuda", generator=g)
    gxh = torch.empty(n, h, w, 16, dtype=torch.bfloat16, device="cuda")
    part = torch.empty(17 * ((n * h * w + 4095) // 4096), device="cuda")
    gwb = torch.empty(17, device="cuda")
    check(lib.fwi_unet_head_bwd(ptr(x16), ptr(hw), ptr(gout), ptr(gxh), ptr(part), ptr(gwb), n, h, w, st), "head_bwd")
    assert _relerr(gwb[:16], (x16.float() * gout[..., None]).sum((0, 1, 2))) < 1e-5
    assert abs(float(gwb[16] - gout.sum())) < 1e-4 * float(gout.abs().sum())
    assert (gxh.float() - _bf(gout[..., None] * hw)).abs().max() <= 1e-2 * float((gout[..., None] * hw).abs().max())


def _torch_unet(net, planes):
    """fp32 torch model of seispie_b200.unet.UNet with the same weights,
    activations rounded to bf16 where the kernels store them
    (straight-through in backward)."""
    from seispie_b200.unet import LAYERS
    P = {}
    for name, c0, c1, co in LAYERS:
        P[name] = (_torch_w(_bf(net.view(name + ".w")).reshape(-1), co, c0 + c1).detach().requires_grad_(True),
                   net.view(name + ".b").detach().clone().requires_grad_(True))

    def rnd(t):
        return t + (_bf(t) - t).detach()

    def conv(name, x):
        w, b = P[name]
        return rnd(F.relu(F.conv2d(x, w, b, padding=1)))

    x = rnd(torch.cat([planes, torch.zeros(planes.shape[0], 13, *planes.shape[2:], device="cuda")], 1))
    e1 = conv("e1b", conv("e1a", x))
    e2 = conv("e2b", conv("e2a", rnd(F.avg_pool2d(e1, 2))))
    e3 = conv("e3b", conv("e3a", rnd(F.avg_pool2d(e2, 2))))
    bb = conv("bb", conv("ba", rnd(F.avg_pool2d(e3, 2))))
    up = lambda t: t.repeat_interleave(2, 2).repeat_interleave(2, 3)  # noqa: E731
    d3 = conv("d3b", conv("d3a", torch.cat([up(bb), e3], 1)))
    d2 = conv("d2b", conv("d2a", torch.cat([up(d3), e2], 1)))
    d1 = conv("d1b", conv("d1a", torch.cat([up(d2), e1], 1)))
    hw = net.view("head.w").detach().clone().requires_grad_(True)
    hb = net.view("head.b").detach().clone().requires_grad_(True)
    out = torch.einsum("nchw,c->nhw", d1, hw) + hb
    return out, P, hw, hb


@pytest.mark.parametrize("h,w,train", [(32, 48, True), (16, 512, False)])
def test_unet_forward_backward_match_torch_and_training_reduces_loss(h, w, train):
    """48 pixels wide: every convolution on the mma.sync kernel; 512 wide:
    every one on the tcgen05 kernel (level widths 512 to 64)."""
    from seispie_b200.unet import LAYERS, UNet
    net = UNet("cuda", seed=1)
    g = torch.Generator(device="cuda").manual_seed(7)
    n = 2
    planes = torch.randn(n, 3, h, w, device="cuda", generator=g)
    target = torch.randn(n, h, w, device="cuda", generator=g)
    out = net.forward(planes)
    ref, P, hw, hb = _torch_unet(net, planes)
    assert _relerr(out, ref) < 2e-2
    loss, gout = net.mse(out, target)
    ref_loss = ((ref - target) ** 2).mean()
    assert abs(float(loss) - float(ref_loss)) < 2e-2 * float(ref_loss)
    net.backward(gout)
    ref_loss.backward()
    for name, c0, c1, co in LAYERS:
        gw_ref = P[name][0].grad
        gw = _torch_w(net.view(name + ".w", net.g), co, c0 + c1)
        if name == "e1a":
            gw, gw_ref = gw[:, :3], gw_ref[:, :3]
        assert _relerr(gw, gw_ref) < 5e-2, name
        assert _relerr(net.view(name + ".b", net.g), P[name][1].grad) < 5e-2, name
    assert _relerr(net.view("head.w", net.g), hw.grad) < 2e-2
    if not train:
        return
    # a few Adam steps on one batch drive the loss down
    l0 = float(loss)
    for _ in range(60):
        out = net.forward(planes)
        loss, gout = net.mse(out, target)
        net.backward(gout)
        net.adam(2e-3)
    assert float(loss) < 0.5 * l0
