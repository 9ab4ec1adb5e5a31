"""The per-subroutine drop-ins (REINITIALIZATION, GRID_COUPLING, TEMP_GRAD,
PRESSURE_CORRECTION) on the GPU against the oracle's routine of the same name, bit for bit,
through the host (numpy) and device (torch) entry points.  The inputs are the states of
boiling columns a few time steps in (phase change active), three columns per batch at
different steps so that their bands and fluxes differ.
"""
import numpy as np
import pytest

from lica_boiling1d_b200 import routines
from lica_boiling1d_b200.column import ColumnProps
from oracle import oracle

pytestmark = pytest.mark.gpu

N, L = 96, 1.0
STEPS = (2, 4, 7)


def _props():
    return ColumnProps(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3)


@pytest.fixture(scope="module")
def states():
    props = _props()
    out = []
    for k, z0 in zip(STEPS, (0.1, 0.12, 0.15)):
        st = oracle.col_init(N, L, z0, props)
        for _ in range(k):
            assert oracle.col_step(st, N, L, props) == 0
        out.append(st)
    return props, out


def _stack(states, key):
    return np.ascontiguousarray(np.stack([s[key] for s in states]))


def _cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("device", [False, True])
def test_reinitialization_bitwise(states, device):
    props, sts = states
    rng = np.random.default_rng(7)
    phi = _stack(sts, "phi")
    layer = _stack(sts, "layer")
    # disturb the band so the pseudo-time iterations have work to do
    phi = phi + np.where(layer > 0, 1e-3 * rng.standard_normal(phi.shape) / N, 0.0)
    ref = phi.copy()
    for c in range(len(sts)):
        oracle.reinitialization(N, L, ref[c], layer[c].copy(), 10)
    if device:
        import torch
        g = _cuda(phi)
        st = routines.reinitialization(N, L, g, _cuda(layer), 10)
        torch.cuda.synchronize()
        got, st = g.cpu().numpy(), st.cpu().numpy()
    else:
        got = phi.copy()
        st = routines.reinitialization(N, L, got, layer, 10)
    assert np.all(st == 0)
    assert not np.array_equal(ref, phi)          # the band moved
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("ini", [0, 1])
@pytest.mark.parametrize("device", [False, True])
def test_grid_coupling_bitwise(states, ini, device):
    _, sts = states
    psif, layer = _stack(sts, "psif"), _stack(sts, "layer")
    cn0, zn0 = _stack(sts, "psi_cn"), _stack(sts, "psi_zn")
    # start from stale fractions so every masked cell has to be recomputed
    cn0 = np.clip(cn0 + 0.01, 0.0, 1.0)
    zn0 = np.clip(zn0 - 0.01, 0.0, 1.0)
    rcn, rzn = cn0.copy(), zn0.copy()
    for c in range(len(sts)):
        oracle.grid_coupling(N, L, ini, psif[c], layer[c], rcn[c], rzn[c])
    if device:
        import torch
        gcn, gzn = _cuda(cn0), _cuda(zn0)
        routines.grid_coupling(N, L, ini, _cuda(psif), _cuda(layer), gcn, gzn)
        torch.cuda.synchronize()
        gcn, gzn = gcn.cpu().numpy(), gzn.cpu().numpy()
    else:
        gcn, gzn = cn0.copy(), zn0.copy()
        routines.grid_coupling(N, L, ini, psif, layer, gcn, gzn)
    np.testing.assert_array_equal(gcn, rcn)
    np.testing.assert_array_equal(gzn, rzn)


@pytest.mark.parametrize("device", [False, True])
def test_temp_grad_bitwise(states, device):
    props, sts = states
    dtconst = 2.0 * (8.0 / 15.0) * sts[0]["scal"][0]
    t, cn = _stack(sts, "t"), _stack(sts, "psi_cn")
    phi, layer = _stack(sts, "phi"), _stack(sts, "layer")
    vol0 = np.array([s["scal"][4] for s in sts])
    refs = [oracle.col_temp_grad(N, L, props, dtconst, t[c], cn[c], phi[c], layer[c], vol0[c])
            for c in range(len(sts))]
    if device:
        import torch
        vol = _cuda(vol0)
        out = routines.temp_grad(N, L, props, dtconst, _cuda(t), _cuda(cn), _cuda(phi), _cuda(layer), vol)
        torch.cuda.synchronize()
        out = {k: v.cpu().numpy() for k, v in out.items()}
    else:
        vol = vol0.copy()
        out = routines.temp_grad(N, L, props, dtconst, t, cn, phi, layer, vol)
    assert np.all(out["status"] == 0)
    for c, (it, mflvs, sfgas, sfgas2, imask, v) in enumerate(refs):
        assert it > 0 and out["iterations"][c] == it
        np.testing.assert_array_equal(out["mflvs"][c], mflvs)
        np.testing.assert_array_equal(out["sfgas"][c], sfgas)
        np.testing.assert_array_equal(out["sfgas2"][c], sfgas2)
        np.testing.assert_array_equal(out["imask"][c], imask)
        assert out["vol_tot_iphs"][c] == v
        assert np.abs(mflvs).max() > 0 and np.abs(sfgas).max() > 0   # phase change at the interface


@pytest.mark.parametrize("device", [False, True])
def test_pressure_correction_bitwise(states, device):
    props, sts = states
    dtconst = 2.0 * (5.0 / 12.0 - 17.0 / 60.0) * sts[1]["scal"][0] + 1e-9
    w, p = _stack(sts, "w"), _stack(sts, "p")
    sfgas = _stack(sts, "sfgas")
    # DENF_ZI = 1 / rho on the faces, from the face liquid fraction
    denf_zi = 1.0 / (1.0 + (props.denr - 1.0) * _stack(sts, "psi_zn"))
    rw, rp = w.copy(), p.copy()
    for c in range(len(sts)):
        oracle.col_pressure_correction(N, L, props, dtconst, rw[c], rp[c], denf_zi[c], sfgas[c])
    if device:
        import torch
        gw, gp = _cuda(w), _cuda(p)
        routines.pressure_correction(N, L, props, dtconst, gw, gp, _cuda(denf_zi), _cuda(sfgas))
        torch.cuda.synchronize()
        gw, gp = gw.cpu().numpy(), gp.cpu().numpy()
    else:
        gw, gp = w.copy(), p.copy()
        routines.pressure_correction(N, L, props, dtconst, gw, gp, denf_zi, sfgas)
    np.testing.assert_array_equal(gw, rw)
    np.testing.assert_array_equal(gp, rp)
    assert rp[:, 1].max() == 0.0 and rp[:, 1].min() == 0.0   # P(1) is the reference level
