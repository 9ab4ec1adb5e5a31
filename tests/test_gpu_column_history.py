"""The 1-D boiling column at its stated configuration, run in full on the GPU.

512 uniform flow cells (1024 refined), density ratio 1000, viscosity ratio 20,
conductivity ratio 25, 10 K superheat (Jakob 0.009), film at 0.1 L as a signed-distance
level set, RK3 at CFL 0.3 for 2000 steps, the 1-D POISSON solved exactly.  The GPU runs
all 2000 steps in one persistent launch and records the reference's per-step interface
history -- the TIME and interface position of 0interface.dat (chphase.f:1419-1438) and
the vapour volume VOL_TOT_IPHS (chphase.f:1457) -- which must equal the oracle's at every
step, bit for bit, as must the final state.
"""
import numpy as np
import pytest

from lica_boiling1d_b200 import column as colmod
from lica_boiling1d_b200.column import ColumnProps, Columns
from oracle import oracle

pytestmark = pytest.mark.gpu

N, Z0, STEPS = 512, 0.1, 2000


def column512_props():
    return ColumnProps(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3)


def oracle_run(props, steps):
    st = oracle.col_init(N, 1.0, Z0, props)
    hist = np.zeros((steps, 4))
    for s in range(steps):
        t0 = float(st["scal"][1])
        assert oracle.col_step(st, N, 1.0, props) == 0, f"oracle step {s + 1}"
        hist[s] = oracle.col_history_record(st, t0)
    return st, hist


def test_config1_history_2000_steps_bitwise():
    import torch
    props = column512_props()
    ref, ref_hist = oracle_run(props, STEPS)
    cols = Columns.film(N, 1.0, [Z0], props).to("cuda")
    hist = torch.full((1, STEPS, 4), float("nan"), dtype=torch.float64, device="cuda")
    colmod.history(hist)
    try:
        status = cols.steps(STEPS, props, threads=256)
        torch.cuda.synchronize()
    finally:
        colmod.history(None)
    assert int(status.max()) == 0
    got = hist[0].cpu().numpy()
    # the vapour film grows: the interface rises and the vapour volume follows it
    assert ref_hist[0, 1] == 0.0 and np.all(ref_hist[1:, 1] > Z0)
    assert ref_hist[-1, 1] > ref_hist[1, 1] and ref_hist[-1, 2] > ref_hist[1, 2]
    for q, name in enumerate(colmod.HISTORY):
        bad = np.flatnonzero(got[:, q] != ref_hist[:, q])
        assert bad.size == 0, f"{name}: first difference at step {bad[0] + 1}: {got[bad[0], q]!r} vs " \
                              f"{ref_hist[bad[0], q]!r}"
    host = cols.to(None)
    for k, v in ref.items():
        assert np.array_equal(host.arrays[k][0], v), f"final state differs in {k}"


def test_history_off_leaves_no_record_and_same_state():
    """The recorder changes nothing in the step: the same steps with and without it give
    the same state; with it off nothing is written."""
    import torch
    props = column512_props()
    a = Columns.film(64, 1.0, [0.1], props).to("cuda")
    b = a.to("cuda")
    hist = torch.full((1, 8, 4), -1.0, dtype=torch.float64, device="cuda")
    colmod.history(hist)
    try:
        a.steps(5, props)
    finally:
        colmod.history(None)
    b.steps(5, props)
    torch.cuda.synchronize()
    h = hist[0].cpu().numpy()
    assert np.all(h[5:] == -1.0) and np.all(h[:5, 3] > 0.0)
    ha, hb = a.to(None), b.to(None)
    for k in ha.arrays:
        assert np.array_equal(ha.arrays[k], hb.arrays[k]), k
    before = hist.clone()
    a.steps(2, props)
    torch.cuda.synchronize()
    assert torch.equal(hist, before)
