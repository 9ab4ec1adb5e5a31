"""CPU restatement of the learned-guess U-Net (test infrastructure: only tests/ use it).

The network is new -- the reference has no learned part -- so this oracle follows the
CUDA implementation (lica_boiling1d_b200/csrc/unet.cu) operation by operation: the same
layer table, parameter layout, BF16 rounding points (inputs, every layer output, every
gradient tensor) and FP32 head, with FP64 accumulation where the GPU accumulates in
FP32.  Forward and backward are written out by hand (no autodiff), so the gradient the
GPU's own kernels produce is checked against an independent derivation.
"""
import numpy as np

# (cin0, cin1, cout, level)
LAYERS = [(16, 0, 32, 0), (32, 0, 32, 0), (32, 0, 64, 1), (64, 0, 64, 1), (64, 0, 128, 2), (128, 0, 128, 2),
          (128, 64, 64, 1), (64, 0, 64, 1), (64, 32, 32, 0), (32, 0, 32, 0)]
HEAD = 32


def bf16(x):
    """Round to BF16 (nearest even, through FP32) and return as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p):
    """Flat FP32 parameter vector -> [(W (cout, 3, 3, ctot), b)], (wh, bh)."""
    out, o = [], 0
    for c0, c1, co, _ in LAYERS:
        ct = c0 + c1
        n = co * 9 * ct
        W = np.asarray(p[o:o + n], dtype=np.float64).reshape(co, 3, 3, ct)
        o += n
        b = np.asarray(p[o:o + co], dtype=np.float64)
        o += co
        out.append((W, b))
    wh = np.asarray(p[o:o + HEAD], dtype=np.float64)
    bh = float(p[o + HEAD])
    return out, (wh, bh)


def param_count():
    return sum(co * 9 * (c0 + c1) + co for c0, c1, co, _ in LAYERS) + HEAD + 1


def _shift(x, dy, dx):
    """x[n, y + dy, x + dx, c] with zeros outside (dy, dx in -1..1)."""
    n, h, w, c = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(h, h - dy)
    xs, xe = max(0, -dx), min(w, w - dx)
    out[:, ys:ye, xs:xe] = x[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def conv(x, W):
    """y[p, co] = sum_{tap, ci} x[p + (dy-1, dx-1), ci] W[co, dy, dx, ci] (no bias)."""
    y = 0.0
    for dy in range(3):
        for dx in range(3):
            y = y + np.einsum("nhwc,oc->nhwo", _shift(x, dy - 1, dx - 1), W[:, dy, dx, :])
    return y


def conv_input_grad(dz, W):
    """gx[q, ci] = sum_{tap, co} dz[q - (dy-1, dx-1), co] W[co, dy, dx, ci]."""
    g = 0.0
    for dy in range(3):
        for dx in range(3):
            g = g + np.einsum("nhwo,oc->nhwc", _shift(dz, 1 - dy, 1 - dx), W[:, dy, dx, :])
    return g


def conv_weight_grad(dz, x):
    """dW[co, dy, dx, ci] = sum_p dz[p, co] x[p + (dy-1, dx-1), ci]."""
    co, ci = dz.shape[-1], x.shape[-1]
    dW = np.zeros((co, 3, 3, ci))
    for dy in range(3):
        for dx in range(3):
            dW[:, dy, dx, :] = np.einsum("nhwo,nhwc->oc", dz, _shift(x, dy - 1, dx - 1))
    return dW


def pool(x):
    return bf16(0.25 * ((x[:, 0::2, 0::2] + x[:, 0::2, 1::2]) + (x[:, 1::2, 0::2] + x[:, 1::2, 1::2])))


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_grad(g):
    return bf16((g[:, 0::2, 0::2] + g[:, 0::2, 1::2]) + (g[:, 1::2, 0::2] + g[:, 1::2, 1::2]))


def forward(params, rho, f, hsq):
    """rho, f: (n, h, w).  Returns (x0, cache)."""
    layers, (wh, bh) = split_params(params)
    Wb = [bf16(W) for W, _ in layers]
    n, h, w = f.shape
    sigma = np.sqrt(np.mean(f.reshape(n, -1) ** 2, axis=1))
    sigma = np.where(sigma > 0, sigma, 1.0)
    x16 = np.zeros((n, h, w, 16))
    x16[..., 0] = bf16(np.log10(rho) / 3.0)
    x16[..., 1] = bf16(f / sigma[:, None, None])

    def L(l, x):
        W, b = layers[l]
        return bf16(np.maximum(conv(x, Wb[l]) + b, 0.0))

    y = [None] * 10
    y[0] = L(0, x16)
    y[1] = L(1, y[0])
    p1 = pool(y[1])
    y[2] = L(2, p1)
    y[3] = L(3, y[2])
    p2 = pool(y[3])
    y[4] = L(4, p2)
    y[5] = L(5, y[4])
    u2 = up(y[5])
    y[6] = L(6, np.concatenate([u2, y[3]], axis=-1))
    y[7] = L(7, y[6])
    u1 = up(y[7])
    y[8] = L(8, np.concatenate([u1, y[1]], axis=-1))
    y[9] = L(9, y[8])
    out = np.einsum("nhwc,c->nhw", y[9], wh) + bh
    x0 = out * sigma[:, None, None] * hsq * rho
    cache = dict(Wb=Wb, wh=wh, sigma=sigma, rho=rho, x16=x16, y=y, p1=p1, p2=p2, u1=u1, u2=u2)
    return x0, cache


def backward(cache, gx0, hsq):
    """Gradient of sum(gx0 * x0) w.r.t. the flat parameter vector."""
    Wb, wh, y = cache["Wb"], cache["wh"], cache["y"]
    gout = gx0 * cache["sigma"][:, None, None] * hsq * cache["rho"]
    grads = [None] * 10
    g_head_w = np.einsum("nhw,nhwc->c", gout, y[9])
    g_head_b = gout.sum()
    g = bf16(gout[..., None] * wh)

    def layer(l, g_out, x):
        dz = np.where(y[l] > 0, g_out, 0.0)
        grads[l] = (conv_weight_grad(dz, x), dz.sum(axis=(0, 1, 2)))
        return bf16(conv_input_grad(dz, Wb[l]))

    g = layer(9, g, y[8])
    gcat = layer(8, g, np.concatenate([cache["u1"], y[1]], axis=-1))
    g_e1b_dec = gcat[..., 64:]
    g = up_grad(gcat[..., :64])
    g = layer(7, g, y[6])
    gcat = layer(6, g, np.concatenate([cache["u2"], y[3]], axis=-1))
    g_e2b_dec = gcat[..., 128:]
    g = up_grad(gcat[..., :128])
    g = layer(5, g, y[4])
    g_p2 = layer(4, g, cache["p2"])
    g = bf16(g_e2b_dec + 0.25 * up(g_p2))
    g = layer(3, g, y[2])
    g_p1 = layer(2, g, cache["p1"])
    g = bf16(g_e1b_dec + 0.25 * up(g_p1))
    g = layer(1, g, y[0])
    layer(0, g, cache["x16"])
    flat = []
    for l in range(10):
        flat.append(grads[l][0].ravel())
        flat.append(grads[l][1])
    flat.append(g_head_w)
    flat.append([g_head_b])
    return np.concatenate(flat)
