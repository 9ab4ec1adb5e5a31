"""Learned initial guess of the pressure solve: the U-Net's tensor-core primitives.

The network is new (the reference has no learned part); its convolutions run on the
tcgen05 tensor cores through lica_unet_conv3x3_device (BF16 NHWC activations, FP32
accumulation)."""
import ctypes as C

from . import native


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def conv3x3(x0, x1, w, bias=None, relu=False, out=None, out_c0=0, want32=False, stream=None):
    """3x3 convolution of contiguous NHWC BF16 CUDA tensors x0 (and x1, concatenated along
    channels) with weights w of shape (cout, 3, 3, c0 + c1); returns (out BF16, FP32 copy or
    None)."""
    import torch
    for t in (x0, x1, w, bias, out):
        if t is not None and not t.is_contiguous():
            raise ValueError("conv3x3 takes contiguous tensors")
    n, h, wd, c0 = x0.shape
    c1 = x1.shape[-1] if x1 is not None else 0
    cout = w.shape[0]
    if out is None:
        out = torch.empty((n, h, wd, cout), dtype=torch.bfloat16, device=x0.device)
    out32 = torch.empty((n, h, wd, out.shape[-1]), dtype=torch.float32, device=x0.device) if want32 else None
    err = torch.zeros(1, dtype=torch.int32, device=x0.device)
    st = native.lib().lica_unet_conv3x3_device(
        _ptr(x0), c0, _ptr(x1), c1, _ptr(w), _ptr(bias), n, h, wd, cout, int(bool(relu)), _ptr(out), _ptr(out32),
        out.shape[-1], out_c0, _ptr(err), C.c_void_p(stream or torch.cuda.current_stream().cuda_stream))
    native.check(st, "lica_unet_conv3x3_device")
    if int(err.item()):
        raise native.LicaError(5, "lica_unet_conv3x3_device: a bounded wait ran out")
    return out, out32
