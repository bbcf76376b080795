"""The learned surrogate: a six-layer convolutional encoder-decoder whose forward and
backward passes run on the library's BF16 tensor-core kernels (hyd_conv_forward,
hyd_conv_wgrad, hyd_bias_grad, hyd_mse_grad).  PyTorch holds the FP32 master weights,
runs Adam and drives the loop; it computes none of the convolutions.  No reference
counterpart (the reference has no learned part).

Network (width 48, 3 x 3 kernels, NHWC BF16 activations, FP32 accumulation):
    L1  same size   6 -> 48  ReLU        input: bed, roughness, upstream Q, downstream stage,
                                          and the cell's along-flow and cross coordinates
    L2  stride-2 down  48 -> 48  ReLU
    L3  same size  48 -> 48  ReLU       (half resolution)
    L4  stride-2 up    48 -> 48  ReLU
    L5  same size  48 -> 48  ReLU
    L6  same size  48 -> 3              output: u, v, z (FP32), normalised
A layer maps output pixel p and tap t = 3 (dy + 1) + (dx + 1) to an input pixel (the
HYD_CONV_* mappings of include/hydist_b200.h); its data gradient is the adjoint mapping
with the channel-transposed weights, fused with the ReLU derivative of its input.
"""
import ctypes
import math

import numpy as np

from . import lib as hlib

CONV_SAME, CONV_SAME_ADJ, CONV_DOWN, CONV_UP = 0, 1, 2, 3
ADJOINT = {CONV_SAME: CONV_SAME_ADJ, CONV_DOWN: CONV_UP, CONV_UP: CONV_DOWN}
# inputs: bed, roughness, upstream Q, downstream stage, and the along-flow and cross
# coordinates (the levels depend on the distance to the stage edge); outputs u, v, z
IN_CH, OUT_CH, WIDTH = 6, 3, 48
CIN_PAD = 16  # input channels padded to the kernels' 16-channel K step

# (mode, cin, cout, relu): the six layers
LAYERS = [
    (CONV_SAME, IN_CH, WIDTH, True),
    (CONV_DOWN, WIDTH, WIDTH, True),
    (CONV_SAME, WIDTH, WIDTH, True),
    (CONV_UP, WIDTH, WIDTH, True),
    (CONV_SAME, WIDTH, WIDTH, True),
    (CONV_SAME, WIDTH, OUT_CH, False),
]


def pad16(c):
    return (c + 15) // 16 * 16


def _bind():
    lib = hlib.load()
    P, I, L, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
    lib.hyd_conv_forward.restype = I
    lib.hyd_conv_forward.argtypes = [P, I, I, I, I, P, P, I, I, I, I, P, P, I, I, I, P, P]
    lib.hyd_conv_wgrad.restype = I
    lib.hyd_conv_wgrad.argtypes = [P, I, I, I, I, I, P, I, I, I, I, P, P, P]
    lib.hyd_bias_grad.restype = I
    lib.hyd_bias_grad.argtypes = [P, L, I, I, P, P]
    lib.hyd_mse_grad.restype = I
    lib.hyd_mse_grad.argtypes = [P, P, P, L, I, I, F, P, P, P]
    return lib


_pack_index = {}


def pack_index(ncol, cinp, device):
    """Element positions of the packed weight image: for output column n and K index
    k = t cinp + c, element (n, k) of K step s = k // 16 lies at
    s ncol 16 + (n // 8) 128 + (kk // 8) 64 + (n % 8) 8 + kk % 8 (kk = k % 16)."""
    key = (ncol, cinp, str(device))
    if key not in _pack_index:
        import torch
        n = torch.arange(ncol, device=device)[:, None]
        k = torch.arange(9 * cinp, device=device)[None, :]
        s, kk = k // 16, k % 16
        pos = s * (ncol * 16) + (n // 8) * 128 + (kk // 8) * 64 + (n % 8) * 8 + kk % 8
        _pack_index[key] = pos.reshape(-1)
    return _pack_index[key]


def pack_weights(w, ncol, cinp):
    """w: FP32 [nout][9][cin] -> the BF16 shared-memory image for ncol output columns and
    cinp (>= cin) input channels per pixel."""
    import torch
    nout, _, cin = w.shape
    full = torch.zeros((ncol, 9, cinp), dtype=torch.float32, device=w.device)
    full[:nout, :, :cin] = w
    img = torch.empty(ncol * 9 * cinp, dtype=torch.bfloat16, device=w.device)
    img[pack_index(ncol, cinp, w.device)] = full.reshape(-1).to(torch.bfloat16)
    return img


def out_size(mode, H, W, full=None):
    if mode == CONV_DOWN:
        return (H + 1) // 2, (W + 1) // 2
    if mode == CONV_UP:
        return full
    return H, W


class Surrogate:
    """The network on one device: FP32 master weights w[l] ([cout][9][cin]) and biases b[l],
    Adam state, and forward / backward passes through the tensor-core kernels."""

    def __init__(self, device=0, seed=0):
        import torch
        self.lib = _bind()
        self.dev = torch.device("cuda", device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.w, self.b = [], []
        for mode, cin, cout, relu in LAYERS:
            std = math.sqrt(2.0 / (9 * cin)) if relu else math.sqrt(1.0 / (9 * cin))
            self.w.append((torch.randn((cout, 9, cin), generator=g) * std).to(self.dev))
            self.b.append(torch.zeros(cout, device=self.dev))
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.m = [torch.zeros_like(p) for p in self.params()]
        self.v = [torch.zeros_like(p) for p in self.params()]
        self.t = 0

    def params(self):
        return self.w + self.b

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _check(self, rc, what):
        if rc != 0:
            raise hlib.HydError("%s failed (%d): %s" % (what, rc, self.lib.hyd_last_error().decode()))

    def conv(self, x, B, H, W, cin, wpk, bias, ncol, nout, mode, relu, Ho, Wo, mask=None, out_f32=False):
        import torch
        y = torch.empty((B, Ho, Wo, nout), dtype=torch.float32 if out_f32 else torch.bfloat16, device=self.dev)
        rc = self.lib.hyd_conv_forward(x.data_ptr(), B, H, W, cin, wpk.data_ptr(),
                                       bias.data_ptr() if bias is not None else None, ncol, nout, mode,
                                       1 if relu else 0, mask.data_ptr() if mask is not None else None,
                                       y.data_ptr(), Ho, Wo, 1 if out_f32 else 0, self.err.data_ptr(), self._stream())
        self._check(rc, "hyd_conv_forward")
        return y

    def forward(self, x):
        """x: BF16 [B][H][W][16] (IN_CH input channels, zero padded).  Returns the FP32 output
        [B][H][W][3] and the activations the backward pass needs."""
        B, H, W, _ = x.shape
        acts, dims = [x], [(H, W)]
        h, w_ = H, W
        cur = x
        for l, (mode, cin, cout, relu) in enumerate(LAYERS):
            ncol = pad16(cout)
            cinp = pad16(cin)
            Ho, Wo = out_size(mode, h, w_, full=(H, W))
            wpk = pack_weights(self.w[l], ncol, cinp)
            last = l == len(LAYERS) - 1
            cur = self.conv(cur, B, h, w_, cinp, wpk, self.b[l], ncol, cout, mode, relu, Ho, Wo, out_f32=last)
            h, w_ = Ho, Wo
            acts.append(cur)
            dims.append((h, w_))
        return cur, (acts, dims)

    def backward(self, saved, dy_last):
        """Gradients of the weights and biases from the output gradient dy_last (BF16
        [B][H][W][16], channels beyond 3 zero)."""
        import torch
        acts, dims = saved
        B = acts[0].shape[0]
        gw = [torch.zeros_like(w) for w in self.w]
        gb = [torch.zeros_like(b) for b in self.b]
        dy = dy_last
        for l in range(len(LAYERS) - 1, -1, -1):
            mode, cin, cout, relu = LAYERS[l]
            ncol, cinp = pad16(cout), pad16(cin)
            (Hi, Wi), (Ho, Wo) = dims[l], dims[l + 1]
            x = acts[l]
            # accumulated over the padded input channels (the first layer's 16 for 4), the
            # real ones kept
            full = gw[l] if cinp == cin else torch.zeros((cout, 9, cinp), dtype=torch.float32, device=self.dev)
            rc = self.lib.hyd_conv_wgrad(x.data_ptr(), B, Hi, Wi, cinp, mode, dy.data_ptr(), Ho, Wo, ncol, cout,
                                         full.data_ptr(), self.err.data_ptr(), self._stream())
            self._check(rc, "hyd_conv_wgrad")
            if cinp != cin:
                gw[l].copy_(full[:, :, :cin])
            rc = self.lib.hyd_bias_grad(dy.data_ptr(), B * Ho * Wo, ncol, cout, gb[l].data_ptr(), self._stream())
            self._check(rc, "hyd_bias_grad")
            if l == 0:
                break
            # data gradient, fused with the ReLU derivative of this layer's input
            wt = self.w[l].permute(2, 1, 0).contiguous()  # [cin][9][cout]
            wpk = pack_weights(wt, pad16(cin), ncol)
            dy = self.conv(dy, B, Ho, Wo, ncol, wpk, None, pad16(cin), cin, ADJOINT[mode], False, Hi, Wi, mask=x)
        return gw, gb

    def loss_grad(self, pred, target, weight=None):
        """Mean-squared error over the weighted pixels and the three outputs; returns (loss
        as a device scalar, BF16 output gradient with 16 channels)."""
        import torch
        B, H, W, nc = pred.shape
        npix = B * H * W
        dy = torch.empty((B, H, W, 16), dtype=torch.bfloat16, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        denom = float(weight.sum().item()) * nc if weight is not None else float(npix * nc)
        rc = self.lib.hyd_mse_grad(pred.data_ptr(), target.data_ptr(), weight.data_ptr() if weight is not None else None,
                                   npix, nc, 16, 1.0 / max(denom, 1.0), dy.data_ptr(), loss.data_ptr(),
                                   self._stream())
        self._check(rc, "hyd_mse_grad")
        return loss, dy

    def adam(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        """One Adam step on the FP32 masters (PyTorch elementwise ops: the training loop)."""
        import torch
        self.t += 1
        with torch.no_grad():
            for p, g, m, v in zip(self.params(), grads, self.m, self.v):
                m.mul_(b1).add_(g, alpha=1 - b1)
                v.mul_(b2).addcmul_(g, g, value=1 - b2)
                mh = m / (1 - b1 ** self.t)
                vh = v / (1 - b2 ** self.t)
                p.sub_(lr * mh / (vh.sqrt() + eps))

    def check_errors(self):
        if int(self.err.item()) != 0:
            raise hlib.HydError("a tensor-core wait timed out in the surrogate kernels")

    def state_dict(self):
        return {"w": [w.cpu() for w in self.w], "b": [b.cpu() for b in self.b]}

    def load_state_dict(self, d):
        for l in range(len(LAYERS)):
            self.w[l].copy_(d["w"][l].to(self.dev))
            self.b[l].copy_(d["b"][l].to(self.dev))


def _bf16_rounding():
    """An autograd function rounding its input to BF16 in the forward pass (out=True: the
    value passes unrounded) and its gradient to BF16 in the backward pass: the points where
    the kernels store BF16 (each layer's activation; each layer's pre-activation gradient,
    which the data-gradient kernel writes after the ReLU mask; the loss gradient)."""
    import torch

    class RoundBF16(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, out):
            return x if out else x.to(torch.bfloat16).float()

        @staticmethod
        def backward(ctx, g):
            return g.to(torch.bfloat16).float(), None

    return RoundBF16.apply


def reference_forward(w, b, x, bf16=False):
    """The same network in plain PyTorch FP32 (any device; used on the CPU as the gradient
    check): x [B][H][W][IN_CH] FP32, w[l] [cout][9][cin], b[l] [cout].  Returns
    [B][H][W][3].  bf16: round the activations and the gradients to BF16 where the kernels
    store them, so that only the FP32 accumulation order differs from the GPU passes."""
    import torch
    import torch.nn.functional as F
    rnd = _bf16_rounding() if bf16 else None
    B, H, W, _ = x.shape
    cur = x.permute(0, 3, 1, 2)
    for l, (mode, cin, cout, relu) in enumerate(LAYERS):
        k = w[l].reshape(cout, 3, 3, cin).permute(0, 3, 1, 2)  # [cout][cin][ky][kx], tap t = 3 ky + kx
        if mode == CONV_SAME:
            cur = F.conv2d(cur, k, b[l], padding=1)
        elif mode == CONV_DOWN:
            cur = F.conv2d(cur, k, b[l], stride=2, padding=1)
        else:  # CONV_UP: y[o] = sum_t x[(o - d_t) / 2] w[t], the transposed stride-2 convolution
            hi, wi = cur.shape[2], cur.shape[3]
            cur = F.conv_transpose2d(cur, k.transpose(0, 1), b[l], stride=2, padding=1,
                                     output_padding=(H - (2 * hi - 1), W - (2 * wi - 1)))
        if relu:
            cur = F.relu(cur)
        if rnd is not None:
            cur = rnd(cur, l == len(LAYERS) - 1)
    return cur.permute(0, 2, 3, 1)
