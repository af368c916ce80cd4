"""A 4-level BF16 U-Net on the library's own convolution kernels.

Channels 16-32-64-128, two 3x3 convolutions with ReLU per level, 2x2
average pooling down, nearest 2x upsampling up, skip connections fed to the
decoder convolutions as a second input (no concatenated copy), a 1x1 head to
one FP32 output channel.  Weights and activations are bf16, accumulation and
gradients FP32 (``fwi_unet_*`` in include/seispie_b200.h).  Every forward,
backward and Adam step is a sequence of those kernels on the current stream;
torch only owns the buffers.

Images are [n, h, w] with h and w multiples of 8 (three pooling levels); the
input has 3 channels, packed into 16 for the tensor-core convolutions.
"""
from __future__ import annotations


import numpy as np
import torch

from . import _lib
from .engine import check, ptr, stream_handle

CH = (16, 32, 64, 128)
# (name, input channels of in0, of in1 (skip), output channels)
LAYERS = (
    ("e1a", 16, 0, 16), ("e1b", 16, 0, 16),
    ("e2a", 16, 0, 32), ("e2b", 32, 0, 32),
    ("e3a", 32, 0, 64), ("e3b", 64, 0, 64),
    ("ba", 64, 0, 128), ("bb", 128, 0, 128),
    ("d3a", 128, 64, 64), ("d3b", 64, 0, 64),
    ("d2a", 64, 32, 32), ("d2b", 32, 0, 32),
    ("d1a", 32, 16, 16), ("d1b", 16, 0, 16),
)


def _align8(n: int) -> int:
    return (n + 7) // 8 * 8


class UNet:
    """Parameters live in one flat FP32 vector (master weights, Adam moments,
    gradients) with a bf16 copy that the kernels read; each layer's weights
    and bias are views at 8-element-aligned offsets."""

    def __init__(self, device="cuda", seed: int = 0):
        self.device = torch.device(device)
        self.lib = _lib.load()
        self.offsets = {}
        off = 0
        for name, c0, c1, co in LAYERS:
            self.offsets[name + ".w"] = (off, (9, co, c0 + c1))
            off = _align8(off + 9 * co * (c0 + c1))
            self.offsets[name + ".b"] = (off, (co,))
            off = _align8(off + co)
        self.offsets["head.w"] = (off, (16,))
        off = _align8(off + 16)
        self.offsets["head.b"] = (off, (1,))
        off = _align8(off + 1)
        self.size = off
        dev = self.device
        self.w = torch.zeros(off, dtype=torch.float32, device=dev)
        self.wb = torch.zeros(off, dtype=torch.bfloat16, device=dev)
        self.g = torch.zeros(off, dtype=torch.float32, device=dev)
        self.m = torch.zeros(off, dtype=torch.float32, device=dev)
        self.v = torch.zeros(off, dtype=torch.float32, device=dev)
        self.step = 0
        self.init_weights(seed)

    # ------------------------------------------------------------ parameters
    def view(self, name: str, t: torch.Tensor | None = None) -> torch.Tensor:
        o, shape = self.offsets[name]
        n = int(np.prod(shape))
        return (self.w if t is None else t)[o:o + n].view(shape)

    def init_weights(self, seed: int) -> None:
        """He-normal 3x3 weights (fan-in 9 x real input channels), zero biases,
        a small head."""
        rng = np.random.default_rng(seed)
        w = np.zeros(self.size, np.float32)
        for name, c0, c1, co in LAYERS:
            o, shape = self.offsets[name + ".w"]
            real_in = 3 if name == "e1a" else c0 + c1
            a = rng.standard_normal(shape).astype(np.float32) * np.sqrt(2.0 / (9 * real_in))
            if name == "e1a":
                a[:, :, 3:] = 0.0  # packed input channels past the third are zero
            w[o:o + a.size] = a.ravel()
        o, _ = self.offsets["head.w"]
        w[o:o + 16] = rng.standard_normal(16).astype(np.float32) * 0.1
        self.load_flat(w)

    def load_flat(self, w: np.ndarray) -> None:
        self.w.copy_(torch.as_tensor(np.asarray(w, np.float32)))
        self.wb.copy_(self.w.to(torch.bfloat16))

    def state(self) -> dict:
        return dict(w=self.w.cpu().numpy(), step=self.step)

    def save(self, path: str, optimizer_state: bool = True, **meta) -> None:
        """Weights (and, unless optimizer_state is False, the Adam state);
        meta: scalar facts stored beside them (training target, suggested
        number of learned iterations)."""
        extra = dict(m=self.m.cpu().numpy(), v=self.v.cpu().numpy(), step=self.step) if optimizer_state else {}
        np.savez_compressed(path, w=self.w.cpu().numpy(), **extra, **meta)

    @classmethod
    def load(cls, path: str, device="cuda") -> "UNet":
        z = np.load(path)
        net = cls(device)
        net.load_flat(z["w"])
        if "m" in z:
            net.m.copy_(torch.as_tensor(z["m"]))
            net.v.copy_(torch.as_tensor(z["v"]))
            net.step = int(z["step"])
        net.meta = {k: z[k].item() for k in ("target", "learned_iterations") if k in z}
        return net

    # ----------------------------------------------------------- kernels
    def _act(self, n, h, w, c):
        return torch.empty((n, h, w, c), dtype=torch.bfloat16, device=self.device)

    def _conv(self, name, x0, x1, out, n, h, w, relu=True):
        _, c0, c1, co = next(L for L in LAYERS if L[0] == name)
        check(self.lib.fwi_unet_conv3x3(ptr(x0), c0, ptr(x1), c1, ptr(self.view(name + ".w", self.wb)),
                                        ptr(self.view(name + ".b")), co, ptr(out), co, None, 0, n, h, w, int(relu),
                                        stream_handle(None)), "fwi_unet_conv3x3")
        return out

    def forward(self, planes: torch.Tensor) -> torch.Tensor:
        """planes [n, 3, h, w] FP32 -> output [n, h, w] FP32; keeps the
        activations for backward()."""
        n, c, h, w = planes.shape
        if c != 3 or h % 8 or w % 8:
            raise ValueError("UNet input must be [n, 3, h, w] with h, w multiples of 8")
        lib, st = self.lib, stream_handle(None)
        a = {}
        x0 = self._act(n, h, w, 16)
        planes = planes.contiguous()  # held while the queued kernel reads it
        check(lib.fwi_unet_pack(ptr(planes), ptr(x0), n, h, w, st), "fwi_unet_pack")
        a["x0"] = x0
        hs = [(h, w), (h // 2, w // 2), (h // 4, w // 4), (h // 8, w // 8)]
        prev = x0
        for lvl, (name_a, name_b) in enumerate((("e1a", "e1b"), ("e2a", "e2b"), ("e3a", "e3b"), ("ba", "bb"))):
            hh, ww = hs[lvl]
            if lvl > 0:
                p = self._act(n, hh, ww, CH[lvl - 1])
                check(lib.fwi_unet_pool2(ptr(prev), ptr(p), CH[lvl - 1], n, 2 * hh, 2 * ww, st), "fwi_unet_pool2")
                a["p%d" % lvl] = p
                prev = p
            ya = self._conv(name_a, prev, None, self._act(n, hh, ww, CH[lvl]), n, hh, ww)
            yb = self._conv(name_b, ya, None, self._act(n, hh, ww, CH[lvl]), n, hh, ww)
            a[name_a], a[name_b] = ya, yb
            prev = yb
        for lvl, (name_a, name_b, skip) in zip((2, 1, 0), (("d3a", "d3b", "e3b"), ("d2a", "d2b", "e2b"),
                                                           ("d1a", "d1b", "e1b"))):
            hh, ww = hs[lvl]
            u = self._act(n, hh, ww, CH[lvl + 1])
            check(lib.fwi_unet_up2(ptr(prev), ptr(u), CH[lvl + 1], n, hh // 2, ww // 2, st), "fwi_unet_up2")
            a["u%d" % lvl] = u
            ya = self._conv(name_a, u, a[skip], self._act(n, hh, ww, CH[lvl]), n, hh, ww)
            yb = self._conv(name_b, ya, None, self._act(n, hh, ww, CH[lvl]), n, hh, ww)
            a[name_a], a[name_b] = ya, yb
            prev = yb
        out = torch.empty((n, h, w), dtype=torch.float32, device=self.device)
        check(lib.fwi_unet_head(ptr(prev), ptr(self.view("head.w")), ptr(self.view("head.b")), ptr(out), n, h, w, st),
              "fwi_unet_head")
        self.acts, self.shape = a, (n, h, w)
        return out

    def _conv_bwd(self, name, gy, x0, x1, n, h, w, need_input_grad=True, gx1=None):
        """Backward of one ReLU 3x3 layer given dL/d(output) gy (bf16,
        modified in place by the ReLU mask).  Writes the layer's weight and
        bias gradients into self.g; returns dL/d(in0) (and writes dL/d(in1)
        into gx1 when the layer has a skip input)."""
        lib, st = self.lib, stream_handle(None)
        _, c0, c1, co = next(L for L in LAYERS if L[0] == name)
        y = self.acts[name]
        check(lib.fwi_unet_relu_bwd(ptr(gy), ptr(y), gy.numel(), st), "fwi_unet_relu_bwd")
        need = lib.fwi_unet_wgrad_partials(co, c0 + c1, n, h, w)
        if self._part.numel() < need:
            self._part = torch.empty(need, dtype=torch.float32, device=self.device)
        check(lib.fwi_unet_conv3x3_wgrad(ptr(gy), co, ptr(x0), c0, ptr(x1), c1, n, h, w, ptr(self._part),
                                         ptr(self.view(name + ".w", self.g)), ptr(self.view(name + ".b", self.g)), st),
              "fwi_unet_conv3x3_wgrad")
        if not need_input_grad:
            return None
        wd = torch.empty(9 * co * (c0 + c1), dtype=torch.bfloat16, device=self.device)
        check(lib.fwi_unet_flip_weights(ptr(self.view(name + ".w", self.wb)), ptr(wd), co, c0 + c1, st),
              "fwi_unet_flip_weights")
        gx0 = self._act(n, h, w, c0)
        check(lib.fwi_unet_conv3x3(ptr(gy), co, None, 0, ptr(wd), None, c0 + c1, ptr(gx0), c0, ptr(gx1), c1, n, h, w,
                                   0, st), "fwi_unet_conv3x3 (data gradient)")
        return gx0

    def backward(self, gout: torch.Tensor) -> None:
        """dL/d(output) [n, h, w] FP32 -> parameter gradients in self.g."""
        lib, st = self.lib, stream_handle(None)
        n, h, w = self.shape
        a = self.acts
        self._part = torch.empty(max(17 * ((n * h * w + 4095) // 4096), 1), dtype=torch.float32, device=self.device)
        hs = [(h, w), (h // 2, w // 2), (h // 4, w // 4), (h // 8, w // 8)]
        g = self._act(n, h, w, 16)
        gout = gout.contiguous()
        check(lib.fwi_unet_head_bwd(ptr(a["d1b"]), ptr(self.view("head.w")), ptr(gout), ptr(g),
                                    ptr(self._part), ptr(self.g[self.offsets["head.w"][0]:]), n, h, w, st),
              "fwi_unet_head_bwd")
        # head.w and head.b are adjacent in the flat vector only through the
        # 17-float result: copy the bias gradient to its slot
        ow, ob = self.offsets["head.w"][0], self.offsets["head.b"][0]
        if ob != ow + 16:
            self.g[ob:ob + 1].copy_(self.g[ow + 16:ow + 17])
        skips = {}
        for lvl, (name_a, name_b, skip) in zip((0, 1, 2), (("d1a", "d1b", "e1b"), ("d2a", "d2b", "e2b"),
                                                           ("d3a", "d3b", "e3b"))):
            hh, ww = hs[lvl]
            g = self._conv_bwd(name_b, g, a[name_a], None, n, hh, ww)
            gskip = self._act(n, hh, ww, CH[lvl])
            gu = self._conv_bwd(name_a, g, a["u%d" % lvl], a[skip], n, hh, ww, gx1=gskip)
            skips[skip] = gskip
            g = self._act(n, hh // 2, ww // 2, CH[lvl + 1])
            check(lib.fwi_unet_up2_bwd(ptr(gu), ptr(g), CH[lvl + 1], n, hh // 2, ww // 2, st), "fwi_unet_up2_bwd")
        for lvl, (name_a, name_b, inp) in zip((3, 2, 1, 0), (("ba", "bb", "p3"), ("e3a", "e3b", "p2"),
                                                             ("e2a", "e2b", "p1"), ("e1a", "e1b", "x0"))):
            hh, ww = hs[lvl]
            if lvl < 3:
                # gradient of this level's output: the skip path plus the pooled path (accumulated)
                gs = skips[name_b]
                check(lib.fwi_unet_pool2_bwd(ptr(g), ptr(gs), CH[lvl], n, hh, ww, 1, st), "fwi_unet_pool2_bwd")
                g = gs
            g = self._conv_bwd(name_b, g, a[name_a], None, n, hh, ww)
            g = self._conv_bwd(name_a, g, a[inp], None, n, hh, ww, need_input_grad=lvl > 0)

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step += 1
        check(self.lib.fwi_unet_adam(ptr(self.w), ptr(self.m), ptr(self.v), ptr(self.g), ptr(self.wb), self.size,
                                     float(lr), float(beta1), float(beta2), float(eps), self.step, stream_handle(None)),
              "fwi_unet_adam")

    def mse(self, out: torch.Tensor, target: torch.Tensor) -> tuple:
        """(loss as a device FP64 scalar, dloss/dout)."""
        gout = torch.empty_like(out)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        part = torch.empty(self.lib.fwi_unet_mse_partials(), dtype=torch.float64, device=self.device)
        target = target.contiguous()
        check(self.lib.fwi_unet_mse(ptr(out), ptr(target), ptr(gout), ptr(loss), ptr(part), out.numel(),
                                    stream_handle(None)), "fwi_unet_mse")
        return loss, gout


def bench(h: int = 2048, w: int = 1024, reps: int = 20) -> list:
    """TFLOP/s of the 3x3 convolution (forward and data gradient on the
    tcgen05 and on the mma.sync kernel, weight gradient) at the four U-Net
    levels of an h x w image (CUDA events, after warm-up)."""
    from .engine import check, ptr, stream_handle
    lib = _lib.load()
    dev = torch.device("cuda")
    st = stream_handle(None)
    out = []
    for lvl, c in enumerate(CH):
        hh, ww = h >> lvl, w >> lvl
        x = torch.randn(1, hh, ww, c, device=dev).to(torch.bfloat16)
        wt = (torch.randn(9 * c * c, device=dev) * 0.05).to(torch.bfloat16)
        wd = torch.empty_like(wt)
        check(lib.fwi_unet_flip_weights(ptr(wt), ptr(wd), c, c, st), "flip")
        y = torch.empty_like(x)
        b = torch.zeros(c, device=dev)
        part = torch.empty(lib.fwi_unet_wgrad_partials(c, c, 1, hh, ww), device=dev)
        dw = torch.empty(9 * c * c, device=dev)
        flops = 2.0 * hh * ww * 9 * c * c
        res = dict(level=lvl, image=[hh, ww], channels=c)
        cases = []
        for path, tag in ((0, ""), (1, "_mma_sync")):
            cases += [("fwd" + tag, path, lambda: lib.fwi_unet_conv3x3(ptr(x), c, None, 0, ptr(wt), ptr(b), c, ptr(y), c,
                                                                       None, 0, 1, hh, ww, 1, st)),
                      ("dgrad" + tag, path, lambda: lib.fwi_unet_conv3x3(ptr(y), c, None, 0, ptr(wd), None, c, ptr(x), c,
                                                                         None, 0, 1, hh, ww, 0, st))]
        cases.append(("wgrad", 0, lambda: lib.fwi_unet_conv3x3_wgrad(ptr(x), c, ptr(y), c, None, 0, 1, hh, ww,
                                                                     ptr(part), ptr(dw), None, st)))
        for name, path, fn in cases:
            old = lib.fwi_unet_conv_path(path)
            try:
                for _ in range(3):
                    check(fn(), name)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    fn()
                e1.record()
                torch.cuda.synchronize()
            finally:
                lib.fwi_unet_conv_path(old)
            ms = e0.elapsed_time(e1) / reps
            res[name + "_us"] = round(ms * 1e3, 2)
            res[name + "_tflops"] = round(flops / (ms * 1e-3) / 1e12, 1)
        out.append(res)
    return out


if __name__ == "__main__":
    # python -m seispie_b200.unet [rows columns [repetitions]]
    import json
    import sys
    args = [int(a) for a in sys.argv[1:4]]
    for r in bench(*args):
        print(json.dumps(r))
