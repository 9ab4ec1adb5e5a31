"""GPU level-set transport (lica_gpu_lvs_transport) against the oracle, bit for bit.

Every case runs the same sequence of TRANSPORT + GRID_COUPLING(0) calls through the C ABI
(a batch of columns per call) and through the oracle (column by column), and compares the
whole state after every call: band phi, layers, PSIF, WO, the target volume, PSI_CN,
PSI_ZN and the per-column statistics.  The library is built without FMA contraction and
sums in the reference's order, so the results agree exactly.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DENR = 1605.36   # lica.in density ratio of the shipped case


def coupled_psi(psif):
    n = (psif.shape[0] - 2) // 2
    pc = np.zeros(n + 2)
    pz = np.zeros(n + 2)
    k = np.arange(1, n + 1)
    pc[1:n + 1] = 0.5 * (psif[2 * k - 1] + psif[2 * k])
    pz[2:n + 1] = 0.5 * (psif[2 * k[1:] - 2] + psif[2 * k[1:] - 1])
    for a in (pc, pz):
        a[a < 1e-3] = 0.0
        a[a > 0.999] = 1.0
    pc[0], pc[n + 1] = pc[1], pc[n]
    return pc, pz


def velocity(n, rng, scale):
    """Smooth seeded face velocity: W(1) = 0 at the wall, a random low-mode profile above."""
    z = np.arange(n + 2) / n
    w = scale * (rng.uniform(0.3, 1.0) + 0.3 * np.sin(2 * np.pi * (z * rng.integers(1, 4) + rng.uniform())))
    w[0] = w[1] = 0.0
    return w


def mass_flux(st, rng, amp):
    mf = np.zeros_like(st["phi"])
    band = st["layer"] > 0
    mf[band] = amp * rng.uniform(0.5, 1.0, band.sum())
    return mf


class Case:
    def __init__(self, n, z0s, seed, wscale, iphs, mf_amp, length=1.0):
        self.n, self.length, self.iphs = n, length, iphs
        self.rng = np.random.default_rng(seed)
        self.states = [O.lvs_init(n, length, z0) for z0 in z0s]
        self.pcs, self.pzs = zip(*[coupled_psi(s["psif"]) for s in self.states])
        self.pcs, self.pzs = list(self.pcs), list(self.pzs)
        self.wscale, self.mf_amp = wscale, mf_amp

    def inputs(self):
        ws = np.stack([velocity(self.n, self.rng, self.wscale) for _ in self.states])
        mfs = np.stack([mass_flux(s, self.rng, self.mf_amp) for s in self.states])
        vis = np.array([s["vol_tot_ori"] * (1.0 + self.rng.uniform(0, 2e-4)) for s in self.states])
        return ws, mfs, vis

    def batch(self):
        from lica_boiling1d_b200.levelset import ColumnBatch
        stack = lambda key: np.ascontiguousarray(np.stack([s[key] for s in self.states]))  # noqa: E731
        return ColumnBatch.from_arrays(self.n, self.length, phi=stack("phi"), layer=stack("layer"),
                                       psif=stack("psif"), wo=stack("wo"),
                                       vol_tot_ori=np.array([s["vol_tot_ori"] for s in self.states]),
                                       psi_cn=np.stack(self.pcs), psi_zn=np.stack(self.pzs))

    def oracle_step(self, ws, mfs, vis, **prm):
        stats = []
        for c, st in enumerate(self.states):
            st2, pc, pz, s = O.lvs_transport(st, ws[c], mfs[c], iphs=self.iphs, vol_tot_iphs=vis[c],
                                             psi_cn=self.pcs[c], psi_zn=self.pzs[c], **prm)
            self.states[c], self.pcs[c], self.pzs[c] = st2, pc, pz
            stats.append(s)
        return np.stack(stats)


def compare(case, batch, stats_gpu, stats_orc, status, where):
    assert np.all(status == 0), (where, status)
    for c, st in enumerate(case.states):
        for key in ("phi", "layer", "psif", "wo"):
            a, b = getattr(batch, key)[c], st[key]
            assert np.array_equal(a, b), (where, c, key, np.max(np.abs(a - b)), np.nonzero(a != b)[0][:8])
        assert batch.vol_tot_ori[c] == st["vol_tot_ori"], (where, c, batch.vol_tot_ori[c], st["vol_tot_ori"])
        assert np.array_equal(batch.psi_cn[c], case.pcs[c]), (where, c, "psi_cn")
        assert np.array_equal(batch.psi_zn[c], case.pzs[c]), (where, c, "psi_zn")
        # stats[1:3] are not written when nothing moved (stats[0] = 0)
        n_out = 4 if stats_orc[c][0] > 0 else 1
        assert np.array_equal(stats_gpu[c][:n_out], stats_orc[c][:n_out]), (where, c, stats_gpu[c], stats_orc[c])


def run(case, steps, m0=1, dt=1e-3, mglobal=1):
    from lica_boiling1d_b200 import levelset
    batch = case.batch()
    for i, m in enumerate(range(m0, m0 + steps)):
        ws, mfs, vis = case.inputs()
        prm = dict(denr=DENR, dtconst=dt, first=int(i == 0), m_step=m, mglobal=mglobal)
        status, sg = levelset.transport(batch, ws, mfs, vis, iphs=case.iphs, **prm)
        so = case.oracle_step(ws, mfs, vis, **prm)
        compare(case, batch, sg, so, status, f"step {m}")
    return batch


def test_shipped_column_phase_change():
    """The shipped column (256 flow cells, interface at 0.0607) with phase change, across
    the 50-step mass-correction / band-rebuild trigger."""
    case = Case(256, [0.0607], seed=1, wscale=0.5, iphs=1, mf_amp=0.02)
    run(case, 12, m0=44)


@pytest.mark.parametrize("iphs", [0, 1])
def test_batch_of_columns(iphs):
    """37 columns (not a multiple of the 4 per CTA), interfaces spread over the column,
    velocities large enough for several subcycles and reinitialisation triggers."""
    rng = np.random.default_rng(7 + iphs)
    z0s = rng.uniform(0.05, 0.9, 37)
    case = Case(512, z0s, seed=11 + iphs, wscale=3.0, iphs=iphs, mf_amp=0.05)
    run(case, 8, m0=47)


def test_interface_near_wall_and_top():
    """Bands cut by the k = 1 and k = nf ends (no band cell at k = 1; ghosts from ALPHI_BC)."""
    case = Case(128, [0.008, 0.011, 0.989, 0.996], seed=3, wscale=0.2, iphs=1, mf_amp=0.01)
    run(case, 6, m0=48)


def test_short_columns_whole_window():
    """Columns short enough for the window to hold the whole column and both ghost ends."""
    case = Case(32, [0.3, 0.5, 0.71], seed=5, wscale=0.3, iphs=1, mf_amp=0.01)
    run(case, 6, m0=49)


def test_no_motion_skip_path():
    case = Case(256, [0.2, 0.4], seed=9, wscale=0.0, iphs=0, mf_amp=0.0)
    run(case, 2)


def test_band_overflow_leaves_column_unchanged():
    """A column with two films 150 refined cells apart has a band wider than the window:
    that column reports LICA_BAND_OVERFLOW and keeps its state, the others proceed."""
    from lica_boiling1d_b200 import levelset
    case = Case(256, [0.3, 0.3], seed=13, wscale=0.5, iphs=0, mf_amp=0.0)
    a = O.lvs_init(256, 1.0, 0.3)
    b = O.lvs_init(256, 1.0, 0.3 + 150 / 512)
    two = O.lvs_copy(a)
    mb = b["layer"] > 0
    two["layer"][mb] = b["layer"][mb]
    two["phi"][mb] = -b["phi"][mb]
    case.states[1] = two
    batch = case.batch()
    before = {k: getattr(batch, k).copy() for k in ("phi", "layer", "psif", "wo", "psi_cn", "psi_zn")}
    ws, mfs, vis = case.inputs()
    status, _ = levelset.transport(batch, ws, mfs, vis, iphs=0, denr=DENR, dtconst=1e-3, first=1, m_step=1)
    assert status[0] == 0 and status[1] == 2
    for k, v in before.items():
        assert np.array_equal(getattr(batch, k)[1], v[1]), k
    assert not np.array_equal(batch.phi[0], before["phi"][0])


def test_device_path_matches_host_path():
    import torch
    from lica_boiling1d_b200 import levelset
    case = Case(512, np.linspace(0.1, 0.8, 9), seed=21, wscale=2.0, iphs=1, mf_amp=0.03)
    host = case.batch()
    dev = host.to("cuda")
    for i, m in enumerate(range(48, 53)):
        ws, mfs, vis = case.inputs()
        prm = dict(iphs=1, denr=DENR, dtconst=1e-3, first=int(i == 0), m_step=m)
        sh, stats_h = levelset.transport(host, ws, mfs, vis, **prm)
        tw = torch.as_tensor(ws, device="cuda")
        sd, stats_d = levelset.transport(dev, tw, torch.as_tensor(mfs, device="cuda"),
                                         torch.as_tensor(vis, device="cuda"), **prm)
        torch.cuda.synchronize()
        assert np.array_equal(sd.cpu().numpy(), sh) and np.array_equal(stats_d.cpu().numpy(), stats_h)
    back = dev.to(None)
    for k in ("phi", "layer", "psif", "wo", "vol_tot_ori", "psi_cn", "psi_zn"):
        assert np.array_equal(getattr(back, k), getattr(host, k)), k


@pytest.mark.parametrize("iphs", [0, 1])
def test_stretched_flow_grid(iphs):
    """TRANSPORT + GRID_COUPLING(0) of columns on a wall-clustered flow grid (HYPTAN, gam 1.5):
    VEL_INTP's stencil on the stretched faces and the coupling boxes from GEOM_COUPLING's
    tables, host and device entries, bit for bit against the oracle on the same geometry."""
    import torch
    from lica_boiling1d_b200 import levelset
    from lica_boiling1d_b200.column import ColumnGeometry
    n = 96
    geo = ColumnGeometry.tanh(n, 1.0, 1.5)
    case = Case(n, [0.12, 0.3, 0.62], seed=21 + iphs, wscale=0.4, iphs=iphs, mf_amp=0.05)
    host = case.batch()
    dev = host.to("cuda")
    for i, m in enumerate(range(1, 7)):
        ws, mfs, vis = case.inputs()
        prm = dict(denr=DENR, dtconst=1e-3, first=int(i == 0), m_step=m, mglobal=1)
        st_h, sg_h = levelset.transport(host, ws, mfs, vis, iphs=iphs, geometry=geo, **prm)
        st_d, sg_d = levelset.transport(dev, torch.from_numpy(ws).cuda(), torch.from_numpy(mfs).cuda(),
                                        torch.from_numpy(vis).cuda(), iphs=iphs, geometry=geo, **prm)
        torch.cuda.synchronize()
        stats = []
        for c, st in enumerate(case.states):
            st2, pc, pz, s = O.lvs_transport(st, ws[c], mfs[c], iphs=iphs, vol_tot_iphs=vis[c], psi_cn=case.pcs[c],
                                             psi_zn=case.pzs[c], geo=geo.arrays, **prm)
            case.states[c], case.pcs[c], case.pzs[c] = st2, pc, pz
            stats.append(s)
        compare(case, host, sg_h, np.stack(stats), st_h, f"host step {m}")
        compare(case, dev.to(None), sg_d.cpu().numpy(), np.stack(stats), st_d.cpu().numpy(), f"device step {m}")
