"""CNN preconditioner kernels (include/fwi2d_nn.h) vs a torch float32 reference.

The kernels take bf16 operands and accumulate in float32, so the reference is
torch in float32 on the same bf16-rounded operands: only the summation order
differs (relative error ~1e-6 for the float32 outputs).  The whole U-Net is
checked against a torch replica that rounds its activations to bf16 at the
same places, forward and backward."""
import numpy as np
import pytest

from fwi2d_b200 import api, cnn

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
F = torch.nn.functional


def rel(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


def bf(x):
    return x.to(torch.bfloat16).float()


def nhwc_to_nchw(t, N, H, W, C):
    return t.view(N, H, W, C).permute(0, 3, 1, 2)


def w_to_torch(w, cout, cin):  # [cout, 9, cin] -> [cout, cin, 3, 3]
    return w.view(cout, 3, 3, cin).permute(0, 3, 1, 2)


@pytest.mark.parametrize("N,H,W,Cin,Cout,relu", [(2, 9, 37, 32, 48, 1), (1, 17, 16, 16, 16, 0),
                                                 (3, 5, 70, 192, 64, 1), (1, 33, 21, 96, 32, 0)])
def test_conv_forward_and_gradients(N, H, W, Cin, Cout, relu):
    g = torch.Generator().manual_seed(N * 1000 + Cin)
    x = bf(torch.randn(N, H, W, Cin, generator=g))
    w = torch.randn(Cout, 9, Cin, generator=g) * 0.1
    b = torch.randn(Cout, generator=g) * 0.1
    dev = "cuda"
    xd = x.to(dev).to(torch.bfloat16).contiguous()
    wd = w.to(dev).contiguous()
    bd = b.to(dev)
    w16 = torch.empty(w.numel(), dtype=torch.bfloat16, device=dev)
    wt16 = torch.empty_like(w16)
    L = api.lib()
    assert L.fwi_nn_weight_prep(wd.data_ptr(), Cout, Cin, w16.data_ptr(), wt16.data_ptr(), None) == 0
    out32 = torch.empty(N * H * W * Cout, dtype=torch.float32, device=dev)
    out16 = torch.empty(N * H * W * Cout, dtype=torch.bfloat16, device=dev)
    assert L.fwi_nn_conv3x3(xd.data_ptr(), N, H, W, Cin, w16.data_ptr(), bd.data_ptr(), Cout, relu,
                            out16.data_ptr(), out32.data_ptr(), None) == 0
    torch.cuda.synchronize()
    wb = bf(w)
    xr = nhwc_to_nchw(x, N, H, W, Cin).clone().requires_grad_(True)
    wr = w_to_torch(wb, Cout, Cin).clone().requires_grad_(True)
    ref = F.conv2d(xr, wr, b, padding=1)
    if relu:
        ref = F.relu(ref)
    got = nhwc_to_nchw(out32.cpu(), N, H, W, Cout)
    assert rel(got, ref.detach()) < 1e-5
    assert torch.equal(out16.cpu().float(), bf(out32.cpu()))
    # gradients of a bf16 output gradient
    dy = bf(torch.randn(N, H, W, Cout, generator=g))
    ref.backward(nhwc_to_nchw(dy, N, H, W, Cout) if not relu else nhwc_to_nchw(dy, N, H, W, Cout))
    dyd = dy.to(dev).to(torch.bfloat16).contiguous()
    # relu': the kernels get dpre = dy * (out > 0) from fwi_nn_relu_bwd
    if relu:
        dyf = dy.to(dev).contiguous()
        dpre = torch.empty_like(dyd)
        assert L.fwi_nn_relu_bwd(dyf.data_ptr(), out16.data_ptr(), dyd.numel(), dpre.data_ptr(), None) == 0
        dyd = dpre
    dx = torch.empty(N * H * W * Cin, dtype=torch.float32, device=dev)
    assert L.fwi_nn_conv3x3(dyd.data_ptr(), N, H, W, Cout, wt16.data_ptr(), None, Cin, 0, None, dx.data_ptr(),
                            None) == 0
    part = torch.empty(L.fwi_nn_wgrad_partial_floats(N, H, W, Cin, Cout), dtype=torch.float32, device=dev)
    dw = torch.empty(Cout * 9 * Cin, dtype=torch.float32, device=dev)
    db = torch.empty(Cout, dtype=torch.float32, device=dev)
    assert L.fwi_nn_conv3x3_wgrad(xd.data_ptr(), dyd.data_ptr(), N, H, W, Cin, Cout, part.data_ptr(), dw.data_ptr(),
                                  db.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert rel(nhwc_to_nchw(dx.cpu(), N, H, W, Cin), xr.grad) < 1e-5
    assert rel(w_to_torch(dw.cpu(), Cout, Cin), wr.grad) < 1e-5
    if not relu:
        assert rel(db.cpu(), nhwc_to_nchw(dy, N, H, W, Cout).sum(dim=(0, 2, 3))) < 1e-5


def test_pool_and_upcat():
    dev = "cuda"
    L = api.lib()
    N, H, W, C = 2, 11, 9, 16
    x = bf(torch.randn(N, H, W, C))
    xd = x.to(dev).to(torch.bfloat16).contiguous()
    p = torch.empty(N * (H // 2) * (W // 2) * C, dtype=torch.bfloat16, device=dev)
    assert L.fwi_nn_pool2(xd.data_ptr(), N, H, W, C, p.data_ptr(), None) == 0
    ref = F.avg_pool2d(nhwc_to_nchw(x, N, H, W, C), 2)
    assert rel(nhwc_to_nchw(p.cpu().float(), N, H // 2, W // 2, C), ref) < 4e-3  # bf16 output
    g = torch.randn(N, H // 2, W // 2, C)
    din = torch.full((N * H * W * C,), 7.0, device=dev)
    assert L.fwi_nn_pool2_bwd(g.to(dev).contiguous().data_ptr(), N, H, W, C, din.data_ptr(), 0, None) == 0
    xr = nhwc_to_nchw(x, N, H, W, C).clone().requires_grad_(True)
    F.avg_pool2d(xr, 2).backward(nhwc_to_nchw(g, N, H // 2, W // 2, C))
    assert rel(nhwc_to_nchw(din.cpu(), N, H, W, C), xr.grad) < 1e-6
    # up + concat onto an odd target size
    Hs, Ws, C1, C2, Ht, Wt = 5, 4, 32, 16, 11, 9
    a = bf(torch.randn(N, Hs, Ws, C1))
    s = bf(torch.randn(N, Ht, Wt, C2))
    out = torch.empty(N * Ht * Wt * (C1 + C2), dtype=torch.bfloat16, device=dev)
    assert L.fwi_nn_upcat(a.to(dev).to(torch.bfloat16).contiguous().data_ptr(), Hs, Ws, C1,
                          s.to(dev).to(torch.bfloat16).contiguous().data_ptr(), N, Ht, Wt, C2, out.data_ptr(), None) == 0
    ys = torch.clamp(torch.arange(Ht) // 2, max=Hs - 1)
    xs = torch.clamp(torch.arange(Wt) // 2, max=Ws - 1)
    up = a[:, ys][:, :, xs]
    assert torch.equal(out.cpu().float().view(N, Ht, Wt, C1 + C2), torch.cat([up, s], dim=3))
    gout = torch.randn(N, Ht, Wt, C1 + C2)
    da = torch.empty(N * Hs * Ws * C1, device=dev)
    ds = torch.full((N * Ht * Wt * C2,), 1.0, device=dev)
    assert L.fwi_nn_upcat_bwd(gout.to(dev).contiguous().data_ptr(), N, Ht, Wt, C1, C2, Hs, Ws, da.data_ptr(), 0,
                              ds.data_ptr(), 1, None) == 0
    ar = a.clone().requires_grad_(True)
    torch.cat([ar[:, ys][:, :, xs], s], dim=3).backward(gout)
    assert rel(da.cpu().view(N, Hs, Ws, C1), ar.grad) < 1e-6
    assert rel(ds.cpu().view(N, Ht, Wt, C2), gout[..., C1:] + 1.0) < 1e-6


class TorchUNet(torch.nn.Module):
    """float32 replica of cnn.UNet rounding activations to bf16 where it does."""

    def __init__(self, net):
        super().__init__()
        self.p = {}
        for c in net.layers:
            self.p[c.name] = (torch.nn.Parameter(w_to_torch(bf(c.w.cpu()), c.cout, c.cin).clone()),
                              torch.nn.Parameter(c.b.cpu().clone()))

    def conv(self, name, x, relu=True):
        w, b = self.p[name]
        y = GradBF.apply(F.conv2d(x, w, b, padding=1))
        return RoundBF.apply(F.relu(y)) if relu else y

    def forward(self, x):
        c = self.conv
        a1 = c("e1b", c("e1a", x))
        a2 = c("e2b", c("e2a", RoundBF.apply(F.avg_pool2d(a1, 2))))
        a3 = c("e3b", c("e3a", RoundBF.apply(F.avg_pool2d(a2, 2))))
        a4 = c("bb", c("ba", RoundBF.apply(F.avg_pool2d(a3, 2))))

        def upcat(a, s):
            H, W = s.shape[2:]
            ys = torch.clamp(torch.arange(H) // 2, max=a.shape[2] - 1)
            xs = torch.clamp(torch.arange(W) // 2, max=a.shape[3] - 1)
            return torch.cat([a[:, :, ys][:, :, :, xs], s], dim=1)

        d3 = c("d3b", c("d3a", upcat(a4, a3)))
        d2 = c("d2b", c("d2a", upcat(d3, a2)))
        d1 = c("d1b", c("d1a", upcat(d2, a1)))
        return c("head", d1, relu=False)


class GradBF(torch.autograd.Function):
    """Identity forward; the gradient of a convolution's output is rounded to
    bf16 (the kernels' tensor-core operand) on the way back."""

    @staticmethod
    def forward(ctx, x):
        return x

    @staticmethod
    def backward(ctx, g):
        return bf(g)


class RoundBF(torch.autograd.Function):
    """bf16 rounding forward; backward rounds the gradient to bf16 only where
    the kernels do (after the ReLU mask), so pass it through unchanged."""

    @staticmethod
    def forward(ctx, x):
        return bf(x)

    @staticmethod
    def backward(ctx, g):
        return g


def _chw(t, N, H, W, C):
    return nhwc_to_nchw(t.detach().cpu().float(), N, H, W, C)


def test_unet_forward_backward_vs_torch_replica():
    N, H, W = 2, 37, 23
    net = cnn.UNet(seed=3)
    g = torch.Generator().manual_seed(5)
    x = torch.zeros(N, H, W, 16)
    x[..., :3] = torch.randn(N, H, W, 3, generator=g)
    x = bf(x)
    xd = x.cuda().to(torch.bfloat16).contiguous()
    out = net.forward(xd, N, H, W)
    target = torch.randn(N * H * W, generator=g).cuda()
    net.mse(target)
    for c in net.layers:
        c.gw.zero_()
        c.gb.zero_()
    net.backward(xd, net.dout)
    torch.cuda.synchronize()
    # 1. every layer's backward step, given the kernels' own forward
    #    activations and incoming gradient, matches torch to float32 rounding
    src_grad = {"e1b": net.g["e1a"], "e2b": net.g["e2a"], "e3b": net.g["e3a"], "bb": net.g["ba"],
                "d3a": net.gcat[3], "d3b": net.g["d3a"], "d2a": net.gcat[2], "d2b": net.g["d2a"],
                "d1a": net.gcat[1], "d1b": net.g["d1a"], "head": net.g["d1b"], "e2a": net.gpool[1],
                "e3a": net.gpool[2], "ba": net.gpool[3]}
    for c in net.layers:
        h, w = net.dims[net.level[c.name]]
        xin = _chw(net._input_of(c.name, xd), N, h, w, c.cin)
        if c.name == "head":
            dpre = _chw(net.dout, N, h, w, c.cout)
        else:
            dact = _chw(net.g[c.name], N, h, w, c.cout)
            dpre = bf(dact * (_chw(net.a[c.name], N, h, w, c.cout) > 0))
        wb = w_to_torch(bf(c.w.cpu()), c.cout, c.cin)
        ref_dw = torch.nn.grad.conv2d_weight(xin, wb.shape, dpre, padding=1)
        assert rel(w_to_torch(c.gw.cpu(), c.cout, c.cin), ref_dw) < 1e-5, c.name
        assert rel(c.gb.cpu(), dpre.sum(dim=(0, 2, 3))) < 1e-5, c.name
        if c.name in src_grad:
            ref_dx = torch.nn.grad.conv2d_input(xin.shape, wb, dpre, padding=1)
            if c.name in ("e2a", "e3a", "ba"):  # the pooled map's gradient
                got = _chw(src_grad[c.name], N, h, w, c.cin)
            else:
                got = _chw(src_grad[c.name], N, h, w, c.cin)
            assert rel(got, ref_dx) < 1e-5, c.name
    # 2. end to end against a float32 replica rounding where the kernels do:
    #    equal up to the drift of bf16 rounding flips through 15 layers
    rep = TorchUNet(net)
    y = rep(nhwc_to_nchw(x, N, H, W, 16))
    assert rel(_chw(out, N, H, W, 16)[:, 0], y[:, 0].detach()) < 2e-2
    loss = ((y[:, 0] - target.cpu().view(N, H, W)) ** 2).sum() / (N * H * W)
    assert abs(float(net.loss.item()) / (N * H * W) - float(loss.detach())) / float(loss.detach()) < 2e-2
    loss.backward()
    for c in net.layers:
        wg, _ = rep.p[c.name]
        assert rel(w_to_torch(c.gw.cpu(), c.cout, c.cin), wg.grad) < 0.15, c.name


def test_training_reduces_loss():
    N, H, W = 2, 40, 36
    net = cnn.UNet(seed=1)
    g = torch.Generator().manual_seed(2)
    x = torch.zeros(N, H, W, 16)
    x[..., :3] = torch.randn(N, H, W, 3, generator=g)
    xd = x.cuda().to(torch.bfloat16).contiguous()
    # a target the network can represent: a smooth function of channel 0
    t = F.avg_pool2d(x[..., 0].unsqueeze(1), 3, stride=1, padding=1).reshape(-1).cuda()
    losses = []
    for _ in range(60):
        net.forward(xd, N, H, W)
        net.mse(t)
        net.backward(xd, net.dout)
        net.adam(lr=3e-3)
        losses.append(float(net.loss.item()))
    assert losses[-1] < 0.3 * losses[0], losses[::10]


@pytest.mark.parametrize("N,H,W,Cin,Cout", [(1, 7, 300, 16, 16), (2, 13, 29, 192, 64), (1, 9, 40, 64, 192),
                                            (1, 5, 130, 128, 128)])
def test_tcgen05_and_mma_sync_paths_agree(N, H, W, Cin, Cout):
    """The tcgen05 / TMEM convolution (fwi_nn_conv3x3) and the mma.sync one
    (fwi_nn_conv3x3_mma) give the same float32 sums up to summation order."""
    g = torch.Generator().manual_seed(Cin + Cout)
    x = torch.randn(N * H * W * Cin, generator=g).cuda().to(torch.bfloat16)
    w = (torch.randn(Cout * 9 * Cin, generator=g) * 0.1).cuda().to(torch.bfloat16)
    b = torch.randn(Cout, generator=g).cuda()
    outs = []
    L = api.lib()
    for fn in (L.fwi_nn_conv3x3, L.fwi_nn_conv3x3_mma):
        o = torch.empty(N * H * W * Cout, dtype=torch.float32, device="cuda")
        assert fn(x.data_ptr(), N, H, W, Cin, w.data_ptr(), b.data_ptr(), Cout, 1, None, o.data_ptr(), None) == 0
        outs.append(o)
    assert L.fwi_nn_check() == 0
    assert rel(outs[0], outs[1]) < 1e-5


@pytest.mark.parametrize("N,H,W,Cin,Cout", [(1, 7, 300, 16, 16), (2, 13, 29, 192, 64), (1, 9, 40, 48, 16),
                                            (3, 5, 130, 128, 128), (1, 11, 17, 96, 32)])
def test_tcgen05_and_mma_sync_weight_gradients_agree(N, H, W, Cin, Cout):
    """fwi_nn_conv3x3_wgrad (tcgen05 partials) and fwi_nn_conv3x3_wgrad_mma
    (mma.sync partials) give the same weight and bias gradients."""
    g = torch.Generator().manual_seed(7 * Cin + Cout)
    x = torch.randn(N * H * W * Cin, generator=g).cuda().to(torch.bfloat16)
    dy = torch.randn(N * H * W * Cout, generator=g).cuda().to(torch.bfloat16)
    L = api.lib()
    part = torch.empty(L.fwi_nn_wgrad_partial_floats(N, H, W, Cin, Cout), dtype=torch.float32, device="cuda")
    res = []
    for fn in (L.fwi_nn_conv3x3_wgrad, L.fwi_nn_conv3x3_wgrad_mma):
        dw = torch.empty(Cout * 9 * Cin, dtype=torch.float32, device="cuda")
        db = torch.empty(Cout, dtype=torch.float32, device="cuda")
        assert fn(x.data_ptr(), dy.data_ptr(), N, H, W, Cin, Cout, part.data_ptr(), dw.data_ptr(), db.data_ptr(),
                  None) == 0
        res.append((dw, db))
    assert L.fwi_nn_check() == 0
    assert rel(res[0][0], res[1][0]) < 1e-5
    # the tcgen05 path sums the bias gradient on the tensor cores (an MMA
    # against a block of ones), the mma.sync path per pixel chunk: same sums,
    # another order
    assert rel(res[0][1], res[1][1]) < 1e-6
    # and both against torch
    xr = nhwc_to_nchw(x.float().cpu(), N, H, W, Cin)
    dyr = nhwc_to_nchw(dy.float().cpu(), N, H, W, Cout)
    ref = torch.nn.grad.conv2d_weight(xr, (Cout, Cin, 3, 3), dyr, padding=1)
    assert rel(w_to_torch(res[0][0].cpu(), Cout, Cin), ref) < 1e-5
    assert rel(res[0][1].cpu(), dyr.double().sum(dim=(0, 2, 3))) < 1e-6
