"""The surrogate's tensor-core kernels (GPU): each convolution mapping against PyTorch's
FP32 convolutions on the same BF16-rounded operands, the weight gradient, and the whole
network's loss and gradients checked against the CPU (PyTorch FP32 autograd of the same
network), then a short training run whose loss falls.

Tolerances: the kernels take BF16 operands and accumulate in FP32, so a layer's output
matches the FP32 convolution of the same rounded operands to the BF16 rounding of its
own output (relative 1e-2 of the output's range).  The network's gradients match a CPU
autograd that rounds to BF16 where the kernels store BF16 to 2e-2 relative L2 (the FP32
accumulation order, and the BF16 roundings it flips, differ), and the CPU's FP32-only
gradients to 1e-1 (the BF16 storage's own error).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAYER_TOL = 1e-2
BF16_REF_TOL = 2e-2
GRAD_TOL = 1e-1


def _rel(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-30))


def _ref_conv(x, w, mode, out_hw):
    """PyTorch FP32 convolution with the HYD_CONV_* mapping: x [B][H][W][C], w [n][9][C]."""
    import torch.nn.functional as F
    from hydist import surrogate as S
    B, H, W, C = x.shape
    n = w.shape[0]
    k = w.reshape(n, 3, 3, C).permute(0, 3, 1, 2)
    xc = x.permute(0, 3, 1, 2)
    if mode == S.CONV_SAME:
        y = F.conv2d(xc, k, padding=1)
    elif mode == S.CONV_SAME_ADJ:
        y = F.conv2d(xc, k.flip(2, 3), padding=1)
    elif mode == S.CONV_DOWN:
        y = F.conv2d(xc, k, stride=2, padding=1)
    else:
        Ho, Wo = out_hw
        y = F.conv_transpose2d(xc, k.transpose(0, 1), stride=2, padding=1,
                               output_padding=(Ho - (2 * H - 1), Wo - (2 * W - 1)))
    return y.permute(0, 2, 3, 1)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("cin,ncol,nout", [(48, 48, 48), (16, 48, 48), (48, 16, 3)])
def test_conv_forward_matches_torch(mode, cin, ncol, nout):
    import torch
    from hydist import surrogate as S
    torch.manual_seed(1)
    net = S.Surrogate()
    B, H, W = 2, 37, 45
    if mode == S.CONV_DOWN:
        Ho, Wo = (H + 1) // 2, (W + 1) // 2
    elif mode == S.CONV_UP:
        Ho, Wo = 2 * H - 1, 2 * W  # both output-padding cases
    else:
        Ho, Wo = H, W
    x = torch.randn((B, H, W, cin), device="cuda").to(torch.bfloat16)
    w = torch.randn((nout, 9, cin), device="cuda") * 0.1
    bias = torch.randn(nout, device="cuda") * 0.1
    wpk = S.pack_weights(w, ncol, cin)
    y = net.conv(x, B, H, W, cin, wpk, bias, ncol, nout, mode, False, Ho, Wo, out_f32=True)
    torch.cuda.synchronize()
    net.check_errors()
    ref = _ref_conv(x.float(), w.to(torch.bfloat16).float(), mode, (Ho, Wo)) + bias
    e = float((y - ref).abs().max() / ref.abs().max())
    print("mode %d cin %d ncol %d: max rel %.2e" % (mode, cin, ncol, e))
    assert e <= 1e-3  # FP32 output: only the FP32 accumulation order differs
    # BF16 output with ReLU and a mask
    mask = torch.randn((B, Ho, Wo, nout), device="cuda").to(torch.bfloat16)
    yb = net.conv(x, B, H, W, cin, wpk, bias, ncol, nout, mode, True, Ho, Wo, mask=mask)
    refb = torch.relu(ref) * (mask.float() > 0)
    eb = float((yb.float() - refb).abs().max() / refb.abs().max())
    assert eb <= LAYER_TOL


@pytest.mark.parametrize("mode", [0, 2, 3])
def test_conv_wgrad_matches_torch(mode):
    import torch
    from hydist import surrogate as S
    torch.manual_seed(2)
    net = S.Surrogate()
    B, H, W, cin, nout, ncol = 2, 33, 40, 48, 48, 48
    Ho, Wo = {0: (H, W), 2: ((H + 1) // 2, (W + 1) // 2), 3: (2 * H, 2 * W - 1)}[mode]
    x = torch.randn((B, H, W, cin), device="cuda").to(torch.bfloat16)
    dy = torch.randn((B, Ho, Wo, ncol), device="cuda").to(torch.bfloat16)
    dw = torch.zeros((nout, 9, cin), device="cuda")
    rc = net.lib.hyd_conv_wgrad(x.data_ptr(), B, H, W, cin, mode, dy.data_ptr(), Ho, Wo, ncol, nout, dw.data_ptr(),
                                net.err.data_ptr(), net._stream())
    assert rc == 0
    torch.cuda.synchronize()
    net.check_errors()
    w = torch.zeros((nout, 9, cin), device="cuda", requires_grad=True)
    y = _ref_conv(x.float(), w, mode, (Ho, Wo))
    (y * dy.float()).sum().backward()
    e = _rel(dw, w.grad)
    print("wgrad mode %d: rel L2 %.2e" % (mode, e))
    assert e <= 1e-4


def test_network_gradients_match_cpu():
    """Loss and every weight and bias gradient of the six-layer network against PyTorch
    autograd of the same network on the CPU, from the BF16 input and weights the kernels
    see: (1) with the activations and gradients rounded to BF16 where the kernels store
    them (only the FP32 accumulation order differs: BF16_REF_TOL), (2) in FP32 throughout
    (the BF16 storage's own error, largest in the first layer, whose gradient has passed
    five BF16 data-gradient layers: GRAD_TOL)."""
    import torch
    from hydist import surrogate as S
    torch.manual_seed(3)
    net = S.Surrogate(seed=5)
    B, H, W = 2, 30, 26
    x4 = torch.randn((B, H, W, S.IN_CH)) * 0.5
    tgt = torch.randn((B, H, W, S.OUT_CH)) * 0.2
    x = torch.zeros((B, H, W, 16))
    x[..., :S.IN_CH] = x4
    xg = x.to("cuda").to(torch.bfloat16)
    pred, saved = net.forward(xg)
    loss, dy = net.loss_grad(pred, tgt.to("cuda").contiguous())
    gw, gb = net.backward(saved, dy)
    torch.cuda.synchronize()
    net.check_errors()
    for bf16, tol in ((True, BF16_REF_TOL), (False, GRAD_TOL)):
        wc = [w.detach().cpu().to(torch.bfloat16).float().requires_grad_(True) for w in net.w]
        bc = [b.detach().cpu().clone().requires_grad_(True) for b in net.b]
        out = S.reference_forward(wc, bc, xg.float().cpu()[..., :S.IN_CH], bf16=bf16)
        ref_loss = ((out - tgt) ** 2).mean()
        ref_loss.backward()
        el = abs(float(loss.item()) - float(ref_loss.detach())) / float(ref_loss.detach())
        print("%s reference: loss %.6f vs %.6f (rel %.2e)" % ("BF16-rounding" if bf16 else "FP32",
                                                               float(loss.item()), float(ref_loss.detach()), el))
        assert el <= 2e-2
        for l in range(len(S.LAYERS)):
            ew, eb = _rel(gw[l], wc[l].grad), _rel(gb[l], bc[l].grad)
            print("  layer %d: weight grad rel L2 %.2e, bias grad %.2e" % (l + 1, ew, eb))
            assert ew <= tol and eb <= tol, (bf16, l, ew, eb)


def test_training_reduces_loss():
    """Fifty Adam steps on a fixed smooth target: the loss falls by half."""
    import torch
    from hydist import surrogate as S
    torch.manual_seed(4)
    net = S.Surrogate(seed=6)
    B, H, W = 4, 48, 40
    yy, xx = torch.meshgrid(torch.linspace(0, 1, H), torch.linspace(0, 1, W), indexing="ij")
    x = torch.zeros((B, H, W, 16))
    for b in range(B):
        x[b, ..., 0] = torch.sin(3 * xx + b)
        x[b, ..., 1] = yy
        x[b, ..., 2] = 0.1 * b
        x[b, ..., 3] = 1.0
    tgt = torch.stack([x[..., 0] * 0.5, x[..., 1] * x[..., 0], 0.3 * x[..., 2] + 0.1 * yy], dim=-1)
    xg = x.cuda().to(torch.bfloat16)
    tg = tgt.cuda().contiguous()
    losses = []
    for it in range(50):
        pred, saved = net.forward(xg)
        loss, dy = net.loss_grad(pred, tg)
        gw, gb = net.backward(saved, dy)
        net.adam(gw + gb, lr=3e-3)
        losses.append(float(loss.item()))
    net.check_errors()
    print("loss %.4e -> %.4e" % (losses[0], losses[-1]))
    assert losses[-1] < 0.5 * losses[0]
