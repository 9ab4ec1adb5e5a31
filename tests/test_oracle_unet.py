"""The U-Net oracle's hand-written backward pass against central finite differences of its
own forward pass (BF16 rounding switched off, FP64 throughout): along a random direction
within each parameter tensor, the directional derivative must agree to 1e-6 relative
(step 1e-7, small enough that no ReLU switches inside the difference)."""
import numpy as np

from oracle import unet_ref as U


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(U, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(3)
    n, h, w = 1, 8, 8
    rho = np.where(rng.random((n, h, w)) < 0.3, 1000.0, 1.0)
    f = rng.standard_normal((n, h, w))
    hsq = 1.0 / 64.0
    p = rng.standard_normal(U.param_count()) * 0.05
    gx0 = rng.standard_normal((n, h, w))
    _, cache = U.forward(p, rho, f, hsq)
    g = U.backward(cache, gx0, hsq)
    assert g.shape == p.shape
    segs, o = [], 0
    for l, (c0, c1, co, _) in enumerate(U.LAYERS):
        nw = co * 9 * (c0 + c1)
        segs += [(f"layer {l} weights", o, o + nw), (f"layer {l} bias", o + nw, o + nw + co)]
        o += nw + co
    segs.append(("head", o, p.size))
    eps = 1e-7
    for name, a, b in segs:
        v = np.zeros(p.size)
        v[a:b] = rng.standard_normal(b - a)
        xp, _ = U.forward(p + eps * v, rho, f, hsq)
        xm, _ = U.forward(p - eps * v, rho, f, hsq)
        fd = np.sum(gx0 * (xp - xm)) / (2 * eps)
        an = float(g @ v)
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-12), (name, fd, an)
