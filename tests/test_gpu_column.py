"""Whole RK3 time steps of 1-D boiling columns on the GPU (lica_gpu_column_steps) against
the oracle (oracle/column1d.cpp), bit for bit: after every launch the complete column
state -- W, P, T, PSI_CN, PSI_ZN, the level-set band, PSIF, the phase-change fields MFLVS,
SFGAS, SFGAS2, IMASK_PH, DT/TIME/M/volumes and the step statistics -- must be identical.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def props_for(**kw):
    from lica_boiling1d_b200.column import ColumnProps
    return ColumnProps(**kw)


def compare(dev, refs, where):
    host = dev.to(None)
    for c, ref in enumerate(refs):
        for k, v in ref.items():
            a = host.arrays[k][c]
            assert np.array_equal(a, v), (where, c, k, np.nonzero(a != v)[0][:6], a[a != v][:3], v[a != v][:3])


def run(n, z0s, props, steps, per_call=1):
    import torch
    from lica_boiling1d_b200.column import Columns
    dev = Columns.film(n, 1.0, z0s, props).to("cuda")
    refs = [O.col_init(n, 1.0, z0, props) for z0 in z0s]
    done = 0
    while done < steps:
        k = min(per_call, steps - done)
        status = dev.steps(k, props)
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0, status
        for r in refs:
            for _ in range(k):
                assert O.col_step(r, n, 1.0, props) == 0
        done += k
        compare(dev, refs, f"after step {done}")
    return dev, refs


def test_shipped_column():
    """The shipped lica.in / grid.in column: 256 flow cells, film 0.0607 thick."""
    dev, refs = run(256, [0.0607], props_for(), 6)
    assert refs[0]["stats"][2] > 0          # TEMP_EXTP ran
    assert refs[0]["scal"][4] > refs[0]["scal"][3] - 1e-9


def test_steps_in_one_launch():
    run(256, [0.0607], props_for(), 8, per_call=4)


def test_benchmark_column_config():
    """512 flow cells, film 0.1, density ratio 1000, viscosity ratio 20, conductivity ratio
    25, Jakob number of a 10 K superheat."""
    run(512, [0.1], props_for(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009), 4)


def test_batch_of_columns():
    run(128, [0.05, 0.1, 0.2, 0.35, 0.5], props_for(denr=800.0, jakob=0.02), 6, per_call=2)


def test_without_phase_change():
    run(128, [0.1, 0.3], props_for(iphs=0), 4, per_call=2)


def test_host_path_matches_device_path():
    import torch
    from lica_boiling1d_b200.column import Columns
    props = props_for()
    host = Columns.film(128, 1.0, [0.08, 0.2], props)
    dev = host.to("cuda")
    st_h = host.steps(3, props)
    st_d = dev.steps(3, props)
    torch.cuda.synchronize()
    assert np.array_equal(st_h, st_d.cpu().numpy())
    back = dev.to(None)
    for k in host.arrays:
        assert np.array_equal(host.arrays[k], back.arrays[k]), k


def test_uneven_batch():
    """Columns of different size, length and properties in one launch (longest first),
    each checked against its own oracle run."""
    import torch
    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    n, length, z0, props = uneven_batch(6, seed=3, nmin=16, nmax=160)
    dev = ColumnBatch.films(n, length, z0, props).to("cuda")
    refs = [O.col_init(int(n[c]), float(length[c]), float(z0[c]), props[c]) for c in range(len(n))]
    for call in range(2):
        status = dev.steps(2, threads=64)
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0
        for c, r in enumerate(refs):
            for _ in range(2):
                assert O.col_step(r, int(n[c]), float(length[c]), props[c]) == 0
            got = dev.column(c)
            for k, v in r.items():
                assert np.array_equal(got[k], v), (call, c, k)


def test_long_columns_with_tridiagonal_arrays_in_scratch():
    """Columns longer than the shared-memory cap of a 64-thread launch keep their Thomas
    arrays in global scratch: still bit-identical to the oracle, beside short columns that
    use shared memory in the same launch."""
    import torch
    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    n, length, z0, props = uneven_batch(3, seed=11, nmin=1200, nmax=1600)
    n = np.concatenate([n, [96, 128]])
    length = np.concatenate([length, [96 / 512, 128 / 512]])
    z0 = np.concatenate([z0, [0.1 * 96 / 512 + 0.37 / 512, 0.1 * 128 / 512 + 0.37 / 512]])
    props = list(props) + [props[0], props[1]]
    dev = ColumnBatch.films(n, length, z0, props).to("cuda")
    refs = [O.col_init(int(n[c]), float(length[c]), float(z0[c]), props[c]) for c in range(len(n))]
    start = dev.to("cuda")
    status = dev.steps(2, threads=64)
    torch.cuda.synchronize()
    assert int(status.abs().max()) == 0
    for c, r in enumerate(refs):
        for _ in range(2):
            assert O.col_step(r, int(n[c]), float(length[c]), props[c]) == 0
        got = dev.column(c)
        for k, v in r.items():
            assert np.array_equal(got[k], v), (c, k)
    # the autotuner's other shapes: every column's arrays in scratch (tri_cap = 0) at 128
    # threads, and one-warp CTAs (TEMP_EXTP's two phases in turn on warp 0)
    for th, cap in ((128, 0), (32, -1)):
        other = start.to("cuda")
        status = other.steps(2, threads=th, tri_cap=cap)
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0
        for k in dev.arrays:
            assert torch.equal(dev.arrays[k], other.arrays[k]), (th, k)


@pytest.mark.parametrize("n,gam,z0s,steps", [(64, 1.0, [0.1], 40), (128, 2.0, [0.06, 0.25], 12)])
def test_stretched_column(n, gam, z0s, steps):
    """A flow grid clustered at both walls (HYPTAN, XSI = 0.5): the step reads GEOMETRIC's
    arrays and GEOM_COUPLING's z tables; every launch bit for bit against the oracle on the
    same geometry (40 steps in launches of 1, 3 and 36)."""
    import torch
    from lica_boiling1d_b200.column import ColumnGeometry, Columns
    props = props_for(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3)
    g = ColumnGeometry.tanh(n, 1.0, gam)
    assert np.diff(g.faces).max() / np.diff(g.faces).min() > 1.2
    dev = Columns.film(n, 1.0, z0s, props, geometry=g).to("cuda")
    refs = [O.col_init_geo(n, 1.0, z0, props, g.arrays) for z0 in z0s]
    done = 0
    for k in (1, 3, steps - 4):
        status = dev.steps(k, props)
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0, status
        for r in refs:
            for _ in range(k):
                assert O.col_step_geo(r, n, 1.0, props, g.arrays) == 0
        done += k
        compare(dev, refs, f"stretched, after step {done}")
    assert refs[0]["stats"][3] > 0   # the level set moved


def test_uniform_geometry_tables_match_closed_forms():
    """A 'stretched' column whose faces are uniform takes the table path of every routine
    and must step exactly as the closed-form uniform column does (a power-of-two column,
    whose coordinates are exact either way); the host-array entry
    (lica_gpu_column_steps_geometry) matches the device one."""
    import torch
    from lica_boiling1d_b200.column import ColumnGeometry, Columns
    n = 128
    props = props_for(denr=1000.0, visr=20.0, tcr=25.0, jakob=0.009, cflmax=0.3)
    g = ColumnGeometry(np.arange(n + 1) / n)
    a = Columns.film(n, 1.0, [0.1, 0.3], props).to("cuda")
    b = Columns.film(n, 1.0, [0.1, 0.3], props, geometry=g)
    bd = b.to("cuda")
    sa, sb = a.steps(6, props), bd.steps(6, props)
    sh = b.steps(6, props)
    torch.cuda.synchronize()
    assert int(sa.abs().max()) == 0 and int(sb.abs().max()) == 0 and int(np.abs(sh).max()) == 0
    ha, hb = a.to(None), bd.to(None)
    for k in ha.arrays:
        assert np.array_equal(ha.arrays[k], hb.arrays[k]), k
        assert np.array_equal(b.arrays[k], hb.arrays[k]), k
