"""Tensor-core (tcgen05) 3x3 convolution of the learned-guess U-Net against an FP64 CPU
convolution of the same BF16 inputs and weights: the FP32 output must agree to FP32
accumulation error (|err| <= 2e-5 * sum |x w|), the BF16 output to one BF16 rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref(x, w, bias, relu):
    """x: (n, h, w, c) float64, w: (cout, 3, 3, c) float64 -> (n, h, w, cout) and sum |x w|."""
    n, h, wd, c = x.shape
    xp = np.zeros((n, h + 2, wd + 2, c))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((n, h, wd, w.shape[0]))
    mag = np.zeros_like(out)
    for dy in range(3):
        for dx in range(3):
            patch = xp[:, dy:dy + h, dx:dx + wd, :]
            out += np.einsum("nhwc,oc->nhwo", patch, w[:, dy, dx, :])
            mag += np.einsum("nhwc,oc->nhwo", np.abs(patch), np.abs(w[:, dy, dx, :]))
    out += bias
    if relu:
        out = np.maximum(out, 0.0)
    return out, mag + np.abs(bias)


@pytest.mark.parametrize("n,h,wd,c0,c1,cout,relu", [
    (2, 16, 16, 16, 0, 32, 0),      # 16-channel blocks (32-byte swizzle)
    (1, 16, 16, 32, 0, 32, 1),      # 32-channel blocks (64-byte swizzle)
    (1, 32, 32, 64, 0, 64, 1),      # 64-channel blocks (128-byte swizzle)
    (1, 32, 32, 128, 0, 128, 1),
    (1, 16, 32, 128, 64, 64, 1),    # decoder input: [upsampled, skip]
    (1, 32, 16, 64, 32, 32, 0),     # two sources with different swizzles
    (1, 16, 16, 64, 0, 192, 0),     # N = 192 (256 tensor-memory columns)
    (1, 4, 256, 32, 0, 16, 1),      # 128 x 1 tiles
])
def test_conv3x3_tensor_core(n, h, wd, c0, c1, cout, relu):
    import torch
    from lica_boiling1d_b200 import unet
    g = torch.Generator().manual_seed(7)
    ctot = c0 + c1
    x0 = torch.randn(n, h, wd, c0, generator=g).to(torch.bfloat16)
    x1 = torch.randn(n, h, wd, c1, generator=g).to(torch.bfloat16) if c1 else None
    w = (torch.randn(cout, 3, 3, ctot, generator=g) / np.sqrt(9 * ctot)).to(torch.bfloat16)
    bias = torch.randn(cout, generator=g).float() * 0.1
    out, out32 = unet.conv3x3(x0.cuda(), x1.cuda() if c1 else None, w.cuda(), bias.cuda(), relu=relu,
                              want32=True)
    x = x0.double().numpy() if not c1 else np.concatenate([x0.double().numpy(), x1.double().numpy()], axis=-1)
    ref, mag = _ref(x, w.double().numpy(), bias.double().numpy(), relu)
    got32 = out32.cpu().double().numpy()
    assert np.all(np.abs(got32 - ref) <= 2e-5 * mag + 1e-30), np.abs(got32 - ref).max()
    got16 = out.cpu().double().numpy()
    assert np.all(np.abs(got16 - got32) <= np.abs(got32) * 2.0 ** -8 + 1e-30)
