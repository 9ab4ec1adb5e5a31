"""Initial state of the 1-D column: the library's host-side MAKEFLD + LVSINIT +
GRID_COUPLING(1) (lica_gpu_column_init, no GPU needed) against the oracle, bit for bit,
and the known answers of a planar film (signed distance, vapour volume = film height)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("n,z0", [(256, 0.0607), (512, 0.1), (128, 0.3333), (64, 0.05), (16, 0.5)])
def test_init_matches_oracle(n, z0):
    from lica_boiling1d_b200.column import ColumnProps, Columns
    props = ColumnProps()
    cols = Columns.film(n, 1.0, [z0], props)
    ref = O.col_init(n, 1.0, z0, props)
    for k, v in ref.items():
        if k == "stats":
            continue
        assert np.array_equal(cols.arrays[k][0], v), k
    assert abs(ref["scal"][3] - z0) < 1e-9
    nf = 2 * n
    band = ref["layer"] > 0
    zc = (np.arange(-2, nf + 5) - 0.5) / nf
    assert np.allclose(ref["phi"][band], zc[band] - z0, atol=1e-11)


def test_init_rejects_film_in_first_cell():
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200.column import ColumnProps, Columns
    with pytest.raises(native.LicaError):
        Columns.film(64, 1.0, [0.003], ColumnProps())


def test_uneven_batch_layout_and_init():
    """Packed layout of a batch of uneven columns and each column's initial state against
    the oracle (host code, no GPU)."""
    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    n, length, z0, props = uneven_batch(7, seed=11, nmin=16, nmax=300)
    b = ColumnBatch.films(n, length, z0, props)
    assert b.totals[0] == int((n + 2).sum()) and b.totals[1] == int((2 * n + 7).sum())
    assert b.totals[2] == int((2 * n + 2).sum())
    for c in range(len(n)):
        ref = O.col_init(int(n[c]), float(length[c]), float(z0[c]), props[c])
        got = b.column(c)
        for k, v in ref.items():
            if k != "stats":
                assert np.array_equal(got[k], v), (c, k)


def test_oracle_column_trajectory_is_pinned():
    """The oracle's column state after 0, 3 and 6 steps equals the committed golden
    (tests/golden/make_column_golden.py) bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_column_golden as M
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "column_oracle_n64.npz"))
    for name, z0, kw in M.CASES:
        got = M.trajectory(z0, kw)
        for k, v in got.items():
            assert np.array_equal(v, gold[f"{name}_{k}"]), (name, k)


@pytest.mark.parametrize("n,gam,z0", [(64, 1.0, 0.1), (128, 2.0, 0.25), (96, 1.5, 0.3), (128, 0.0, 0.3)])
def test_stretched_init_matches_oracle(n, gam, z0):
    """lica_gpu_column_init_geometry (host code) on a wall-clustered flow grid (gam = 0:
    uniform faces through the tables) against the oracle, bit for bit; uniform faces of a
    power-of-two column (whose face and centre coordinates are exact) give the closed-form
    column's state exactly."""
    from lica_boiling1d_b200.column import ColumnGeometry, ColumnProps, Columns
    props = ColumnProps(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009)
    g = ColumnGeometry.tanh(n, 1.0, gam) if gam > 0 else ColumnGeometry(np.arange(n + 1) / n)
    cols = Columns.film(n, 1.0, [z0], props, geometry=g)
    ref = O.col_init_geo(n, 1.0, z0, props, g.arrays)
    for k, v in ref.items():
        if k != "stats":
            assert np.array_equal(cols.arrays[k][0], v), k
    if gam == 0:
        u = O.col_init(n, 1.0, z0, props)
        for k in u:
            assert np.array_equal(u[k], ref[k]), k


def test_oracle_table_path_equals_closed_forms():
    """The oracle's stretched step on uniform faces reproduces its uniform step bit for bit
    over 12 steps (the table path of every routine against the pinned closed forms)."""
    from lica_boiling1d_b200.column import ColumnGeometry, ColumnProps
    n, z0 = 64, 0.1
    props = ColumnProps(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3)
    g = ColumnGeometry(np.arange(n + 1) / n)
    a, b = O.col_init(n, 1.0, z0, props), O.col_init_geo(n, 1.0, z0, props, g.arrays)
    for _ in range(12):
        assert O.col_step(a, n, 1.0, props) == 0
        assert O.col_step_geo(b, n, 1.0, props, g.arrays) == 0
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_stretched_geometry_checks():
    """A cell narrower than a refined cell, or faces that do not end at the length, are
    refused (LICA_BAD_ARG), never run."""
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200.column import ColumnGeometry, ColumnProps, Columns
    n = 32
    faces = np.arange(n + 1) / n
    faces[1] = 0.25 / (2 * n)            # first cell a quarter of a refined cell
    with pytest.raises(native.LicaError):
        Columns.film(n, 1.0, [0.3], ColumnProps(), geometry=ColumnGeometry(faces))
    import ctypes as C
    g = ColumnGeometry(np.arange(n + 1) / n)
    st = Columns.empty(1, n, 2.0)
    cs = native.ColState(*[st.arrays[k][0].ctypes.data for k in native.COL_FIELDS])
    gc, cp = g.c(), ColumnProps().c()
    assert native.lib().lica_gpu_column_init_geometry(n, 2.0, 0.3, C.byref(cp), C.byref(gc), C.byref(cs)) == 4   # LICA_BAD_ARG
    with pytest.raises(ValueError):
        Columns.film(n, 2.0, [0.3], ColumnProps(), geometry=g)
