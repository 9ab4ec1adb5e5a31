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


class LearnedGuess:
    """The U-Net initial guess for n images of h x w (lica_unet_*): guess(), train_step(),
    parameter get/set.  Device arrays are contiguous FP64 torch tensors of shape (n, h, w)
    (by: (n, h + 1, w))."""

    def __init__(self, n, h, w, seed=1):
        import numpy as np  # noqa: F401
        self.n, self.h, self.w = n, h, w
        self._h = C.c_void_p()
        native.check(native.lib().lica_unet_create(C.byref(self._h), n, h, w, seed), "lica_unet_create")
        self.nparams = int(native.lib().lica_unet_param_count(self._h))

    def close(self):
        if self._h:
            native.lib().lica_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        import numpy as np
        p = np.empty(self.nparams, dtype=np.float32)
        native.check(native.lib().lica_unet_get_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size),
                     "lica_unet_get_params")
        return p

    def set_params(self, p):
        import numpy as np
        p = np.ascontiguousarray(p, dtype=np.float32)
        native.check(native.lib().lica_unet_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size),
                     "lica_unet_set_params")

    @staticmethod
    def _stream(stream):
        import torch
        return C.c_void_p(stream or torch.cuda.current_stream().cuda_stream)

    def guess(self, rho, f, hsq, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty_like(f)
        native.check(native.lib().lica_unet_guess_device(self._h, _ptr(rho), _ptr(f), float(hsq), _ptr(out),
                                                         self._stream(stream)), "lica_unet_guess_device")
        return out

    def guess_checked(self, rho, f, bx, by, hx, hy, out=None, stream=None):
        """The guess and its relative residual per image; images whose guess is no better
        than zero get x0 = 0.  Returns (x0, rel0 numpy array)."""
        import numpy as np
        import torch
        if out is None:
            out = torch.empty_like(f)
        rel = np.empty(self.n)
        native.check(native.lib().lica_unet_guess_checked_device(
            self._h, _ptr(rho), _ptr(f), _ptr(bx), _ptr(by), float(hx), float(hy), _ptr(out),
            rel.ctypes.data_as(C.POINTER(C.c_double)), self._stream(stream)), "lica_unet_guess_checked_device")
        return out, rel

    def grad(self, rho, f, hsq, gx0, stream=None):
        import numpy as np
        g = np.empty(self.nparams, dtype=np.float32)
        native.check(native.lib().lica_unet_grad_device(self._h, _ptr(rho), _ptr(f), float(hsq), _ptr(gx0),
                                                        g.ctypes.data_as(C.POINTER(C.c_float)), g.size,
                                                        self._stream(stream)), "lica_unet_grad_device")
        return g

    def train_step(self, rho, f, bx, by, hx, hy, lr, p_star=None, stream=None):
        loss = C.c_double()
        native.check(native.lib().lica_unet_train_step_device(self._h, _ptr(rho), _ptr(f), _ptr(bx), _ptr(by),
                                                              _ptr(p_star), float(hx), float(hy), float(lr),
                                                              C.byref(loss), self._stream(stream)),
                     "lica_unet_train_step_device")
        return loss.value
