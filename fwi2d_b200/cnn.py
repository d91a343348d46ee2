"""CNN gradient preconditioner: a 4-level U-Net on (raw gradient, illumination,
model) -> model-update direction, trained on pairs this FD engine makes.

No reference counterpart: the reference's FWI steps along the illumination-
normalised gradient (inversion.cu:111-166, 286-358).  Here the network's
output replaces that direction (fwi_set_direction_dev) before the same
3-point parabolic line search; when the line search does not cut the misfit
the iteration falls back to the plain gradient.

Every operation of the network runs in the project's own kernels
(include/fwi2d_nn.h: 3x3 convolutions and their weight and bias gradients on
the tcgen05 tensor cores, operands loaded by TMA, FP32 accumulators in tensor
memory; pooling, upsampling + skip concatenation, ReLU gradient, MSE, Adam);
torch only allocates device memory.

Architecture (channels c = 16, 32, 64, 128; every conv 3x3, ReLU but the last):
  enc1 3->16->16 | pool | enc2 16->32->32 | pool | enc3 32->64->64 | pool |
  bottom 64->128->128 | up+cat enc3 -> 192->64->64 | up+cat enc2 -> 96->32->32 |
  up+cat enc1 -> 48->16->16 | head 16->16 (channel 0 = direction)
Images are (H = nx, W = nz): pixel p = x * nz + z, the engine's z-fastest order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import api

CH = (16, 32, 64, 128)
IN_CH = 16  # 3 input channels padded to a multiple of 16
OUT_CH = 16  # head output padded; channel 0 is used

# (name, Cin, Cout, relu) in forward order
LAYERS = [
    ("e1a", IN_CH, CH[0], True), ("e1b", CH[0], CH[0], True),
    ("e2a", CH[0], CH[1], True), ("e2b", CH[1], CH[1], True),
    ("e3a", CH[1], CH[2], True), ("e3b", CH[2], CH[2], True),
    ("ba", CH[2], CH[3], True), ("bb", CH[3], CH[3], True),
    ("d3a", CH[3] + CH[2], CH[2], True), ("d3b", CH[2], CH[2], True),
    ("d2a", CH[2] + CH[1], CH[1], True), ("d2b", CH[1], CH[1], True),
    ("d1a", CH[1] + CH[0], CH[0], True), ("d1b", CH[0], CH[0], True),
    ("head", CH[0], OUT_CH, False),
]


def _torch():
    import torch
    return torch


def _lib():
    return api.lib()


def _ok(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc})")


def _p(t) -> int:
    return t.data_ptr()


@dataclass
class Conv:
    name: str
    cin: int
    cout: int
    relu: bool
    w: object = None    # float32 master [cout, 9, cin]
    b: object = None
    gw: object = None
    gb: object = None
    mw: object = None
    vw: object = None
    mb: object = None
    vb: object = None
    w16: object = None  # bf16 [cout, 9, cin]
    wt16: object = None  # bf16 [cin, 9, cout] flipped


class UNet:
    def __init__(self, seed: int = 0, device: str = "cuda", real_in: int = 3):
        torch = _torch()
        self.device = device
        rng = np.random.default_rng(seed)
        self.layers: list[Conv] = []
        for name, cin, cout, relu in LAYERS:
            fan_in = 9 * (real_in if name == "e1a" else cin)
            std = np.sqrt(2.0 / fan_in) if relu else np.sqrt(1.0 / fan_in)
            w = rng.standard_normal((cout, 9, cin)).astype(np.float32) * np.float32(std)
            if name == "e1a":
                w[:, :, real_in:] = 0.0
            if name == "head":
                w[1:] = 0.0
            c = Conv(name, cin, cout, relu)
            c.w = torch.from_numpy(w).to(device)
            c.b = torch.zeros(cout, dtype=torch.float32, device=device)
            for k in ("gw", "mw", "vw"):
                setattr(c, k, torch.zeros_like(c.w))
            for k in ("gb", "mb", "vb"):
                setattr(c, k, torch.zeros_like(c.b))
            c.w16 = torch.empty(c.w.numel(), dtype=torch.bfloat16, device=device)
            c.wt16 = torch.empty(c.w.numel(), dtype=torch.bfloat16, device=device)
            self.layers.append(c)
        self.by_name = {c.name: c for c in self.layers}
        self.step_count = 0
        self.shape = None
        self._prep_weights()

    # -- parameters
    def _prep_weights(self) -> None:
        for c in self.layers:
            _ok(_lib().fwi_nn_weight_prep(_p(c.w), c.cout, c.cin, _p(c.w16), _p(c.wt16), None), "weight prep")

    def state(self) -> dict:
        out = {}
        for c in self.layers:
            out[c.name + ".w"] = c.w.cpu().numpy()
            out[c.name + ".b"] = c.b.cpu().numpy()
        return out

    def load_state(self, st: dict) -> None:
        torch = _torch()
        for c in self.layers:
            c.w.copy_(torch.from_numpy(np.asarray(st[c.name + ".w"], np.float32)))
            c.b.copy_(torch.from_numpy(np.asarray(st[c.name + ".b"], np.float32)))
        self._prep_weights()

    def save(self, path) -> None:
        np.savez(path, **self.state())

    def load(self, path) -> None:
        with np.load(path) as f:
            self.load_state({k: f[k] for k in f.files})

    # -- buffers
    def _alloc(self, N: int, H: int, W: int) -> None:
        if self.shape == (N, H, W):
            return
        torch = _torch()
        dev = self.device
        H1, W1 = H // 2, W // 2
        H2, W2 = H1 // 2, W1 // 2
        H3, W3 = H2 // 2, W2 // 2
        if min(H3, W3) < 1:
            raise ValueError("image too small for a 4-level U-Net")
        self.dims = {1: (H, W), 2: (H1, W1), 3: (H2, W2), 4: (H3, W3)}
        lvl = {"e1a": 1, "e1b": 1, "e2a": 2, "e2b": 2, "e3a": 3, "e3b": 3, "ba": 4, "bb": 4, "d3a": 3, "d3b": 3,
               "d2a": 2, "d2b": 2, "d1a": 1, "d1b": 1, "head": 1}
        self.level = lvl
        bf = torch.bfloat16
        f32 = torch.float32

        def act(level, c, dtype=bf):
            h, w = self.dims[level]
            return torch.zeros(N * h * w * c, dtype=dtype, device=dev)

        self.a = {c.name: act(lvl[c.name], c.cout) for c in self.layers if c.name != "head"}
        self.out32 = act(1, OUT_CH, f32)
        self.pool = {1: act(2, CH[0]), 2: act(3, CH[1]), 3: act(4, CH[2])}
        self.cat = {3: act(3, CH[3] + CH[2]), 2: act(2, CH[2] + CH[1]), 1: act(1, CH[1] + CH[0])}
        # gradients (float32) of activations / concatenations / pooled maps
        self.g = {c.name: act(lvl[c.name], c.cout, f32) for c in self.layers if c.name != "head"}
        self.gcat = {3: act(3, CH[3] + CH[2], f32), 2: act(2, CH[2] + CH[1], f32), 1: act(1, CH[1] + CH[0], f32)}
        self.gpool = {1: act(2, CH[0], f32), 2: act(3, CH[1], f32), 3: act(4, CH[2], f32)}
        # bf16 scratch for one layer's output gradient after the ReLU
        sizes = [N * self.dims[lvl[c.name]][0] * self.dims[lvl[c.name]][1] * c.cout for c in self.layers]
        self.dpre = torch.zeros(max(sizes), dtype=bf, device=dev)
        nmax = max(_lib().fwi_nn_wgrad_partial_floats(N, *self.dims[lvl[c.name]], c.cin, c.cout) for c in self.layers)
        self.partial = torch.zeros(int(nmax), dtype=f32, device=dev)
        self.mse_partial = torch.zeros(256, dtype=torch.float64, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float64, device=dev)
        self.dout = act(1, OUT_CH)
        self.shape = (N, H, W)

    def _input_of(self, name: str, x):
        return {"e1a": x, "e1b": self.a["e1a"], "e2a": self.pool[1], "e2b": self.a["e2a"], "e3a": self.pool[2],
                "e3b": self.a["e3a"], "ba": self.pool[3], "bb": self.a["ba"], "d3a": self.cat[3], "d3b": self.a["d3a"],
                "d2a": self.cat[2], "d2b": self.a["d2a"], "d1a": self.cat[1], "d1b": self.a["d1a"],
                "head": self.a["d1b"]}[name]

    # -- forward
    def forward(self, x, N: int, H: int, W: int):
        """x: NHWC bf16 (C = 16) device tensor; returns out32 ([N,H,W,16] float32)."""
        self._alloc(N, H, W)
        L = _lib()
        d = self.dims

        def conv(name):
            c = self.by_name[name]
            h, w = d[self.level[name]]
            src = self._input_of(name, x)
            if name == "head":
                _ok(L.fwi_nn_conv3x3(_p(src), N, h, w, c.cin, _p(c.w16), _p(c.b), c.cout, 0, None, _p(self.out32),
                                     None), name)
            else:
                _ok(L.fwi_nn_conv3x3(_p(src), N, h, w, c.cin, _p(c.w16), _p(c.b), c.cout, 1, _p(self.a[name]), None,
                                     None), name)

        conv("e1a"); conv("e1b")
        _ok(L.fwi_nn_pool2(_p(self.a["e1b"]), N, *d[1], CH[0], _p(self.pool[1]), None), "pool1")
        conv("e2a"); conv("e2b")
        _ok(L.fwi_nn_pool2(_p(self.a["e2b"]), N, *d[2], CH[1], _p(self.pool[2]), None), "pool2")
        conv("e3a"); conv("e3b")
        _ok(L.fwi_nn_pool2(_p(self.a["e3b"]), N, *d[3], CH[2], _p(self.pool[3]), None), "pool3")
        conv("ba"); conv("bb")
        _ok(L.fwi_nn_upcat(_p(self.a["bb"]), *d[4], CH[3], _p(self.a["e3b"]), N, *d[3], CH[2], _p(self.cat[3]), None),
            "upcat3")
        conv("d3a"); conv("d3b")
        _ok(L.fwi_nn_upcat(_p(self.a["d3b"]), *d[3], CH[2], _p(self.a["e2b"]), N, *d[2], CH[1], _p(self.cat[2]), None),
            "upcat2")
        conv("d2a"); conv("d2b")
        _ok(L.fwi_nn_upcat(_p(self.a["d2b"]), *d[2], CH[1], _p(self.a["e1b"]), N, *d[1], CH[0], _p(self.cat[1]), None),
            "upcat1")
        conv("d1a"); conv("d1b")
        conv("head")
        return self.out32

    # -- backward (after forward on the same x); dout: bf16 [N,H,W,16]
    def backward(self, x, dout) -> None:
        N, H, W = self.shape
        L = _lib()
        d = self.dims

        def layer_bwd(name, d_act, d_src):
            """d_act: float32 gradient of this layer's output activation (None
            for the head, whose output gradient is dout); writes the gradient
            of its input into d_src (float32) unless d_src is None."""
            c = self.by_name[name]
            h, w = d[self.level[name]]
            n = N * h * w * c.cout
            if name == "head":
                dp = dout
            else:
                dp = self.dpre
                _ok(L.fwi_nn_relu_bwd(_p(d_act), _p(self.a[name]), n, _p(dp), None), name + " relu'")
            src = self._input_of(name, x)
            _ok(L.fwi_nn_conv3x3_wgrad(_p(src), _p(dp), N, h, w, c.cin, c.cout, _p(self.partial), _p(c.gw), _p(c.gb),
                                       None), name + " wgrad")
            if d_src is not None:
                _ok(L.fwi_nn_conv3x3(_p(dp), N, h, w, c.cout, _p(c.wt16), None, c.cin, 0, None, _p(d_src), None),
                    name + " dgrad")

        g = self.g
        layer_bwd("head", None, g["d1b"])
        layer_bwd("d1b", g["d1b"], g["d1a"])
        layer_bwd("d1a", g["d1a"], self.gcat[1])
        _ok(L.fwi_nn_upcat_bwd(_p(self.gcat[1]), N, *d[1], CH[1], CH[0], *d[2], _p(g["d2b"]), 0, _p(g["e1b"]), 0, None),
            "upcat1'")
        layer_bwd("d2b", g["d2b"], g["d2a"])
        layer_bwd("d2a", g["d2a"], self.gcat[2])
        _ok(L.fwi_nn_upcat_bwd(_p(self.gcat[2]), N, *d[2], CH[2], CH[1], *d[3], _p(g["d3b"]), 0, _p(g["e2b"]), 0, None),
            "upcat2'")
        layer_bwd("d3b", g["d3b"], g["d3a"])
        layer_bwd("d3a", g["d3a"], self.gcat[3])
        _ok(L.fwi_nn_upcat_bwd(_p(self.gcat[3]), N, *d[3], CH[3], CH[2], *d[4], _p(g["bb"]), 0, _p(g["e3b"]), 0, None),
            "upcat3'")
        layer_bwd("bb", g["bb"], g["ba"])
        layer_bwd("ba", g["ba"], self.gpool[3])
        _ok(L.fwi_nn_pool2_bwd(_p(self.gpool[3]), N, *d[3], CH[2], _p(g["e3b"]), 1, None), "pool3'")
        layer_bwd("e3b", g["e3b"], g["e3a"])
        layer_bwd("e3a", g["e3a"], self.gpool[2])
        _ok(L.fwi_nn_pool2_bwd(_p(self.gpool[2]), N, *d[2], CH[1], _p(g["e2b"]), 1, None), "pool2'")
        layer_bwd("e2b", g["e2b"], g["e2a"])
        layer_bwd("e2a", g["e2a"], self.gpool[1])
        _ok(L.fwi_nn_pool2_bwd(_p(self.gpool[1]), N, *d[1], CH[0], _p(g["e1b"]), 1, None), "pool1'")
        layer_bwd("e1b", g["e1b"], g["e1a"])
        layer_bwd("e1a", g["e1a"], None)

    def mse(self, target, mask=None) -> None:
        """sum_p (mask (out - target))^2 into self.loss (device, FP64) and the
        gradient of that sum / P (the mean) into self.dout."""
        N, H, W = self.shape
        P = N * H * W
        _ok(_lib().fwi_nn_mse(_p(self.out32), OUT_CH, _p(target), _p(mask) if mask is not None else None, P,
                              1.0 / P, _p(self.dout), _p(self.mse_partial), _p(self.loss), None), "mse")

    def adam(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        L = _lib()
        for c in self.layers:
            _ok(L.fwi_nn_adam(_p(c.w), _p(c.gw), _p(c.mw), _p(c.vw), c.w.numel(), lr, b1, b2, eps, self.step_count,
                              None), "adam")
            _ok(L.fwi_nn_adam(_p(c.b), _p(c.gb), _p(c.mb), _p(c.vb), c.b.numel(), lr, b1, b2, eps, self.step_count,
                              None), "adam")
        self._prep_weights()


# ------------------------------------------------------------------ features
def pack(g, il, vp, nz: int, nx: int, out, scratch, v0: float = 3000.0, vs: float = 1.0 / 1000.0) -> None:
    """Device float32 grids (z fastest) -> NHWC bf16 network input (fwi_nn_pack_inputs)."""
    _ok(_lib().fwi_nn_pack_inputs(_p(g), _p(il), _p(vp), nz, nx, v0, vs, _p(scratch), _p(out), None), "pack inputs")


def direction(net: UNet, out32, nz: int, nx: int, dst) -> None:
    _ok(_lib().fwi_nn_unpack(_p(out32), OUT_CH, nz * nx, _p(dst), None), "unpack")
