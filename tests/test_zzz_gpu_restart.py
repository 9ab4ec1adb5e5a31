"""Resuming 1-D columns on the GPU from fld###### restart files: columns stepped on the
device are written from device memory, read back, and stepped again on the device; every
resumed step must equal the oracle's step from the oracle's own reading of the same file,
bit for bit (the complete column state)."""
import numpy as np
import pytest

from oracle import fld as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_resume_on_the_gpu_matches_the_oracle(tmp_path):
    import torch
    from lica_boiling1d_b200 import restart as R
    from lica_boiling1d_b200.column import ColumnProps, Columns
    props = ColumnProps()
    n = 256
    dev = Columns.film(n, 1.0, [0.0607, 0.12], props).to("cuda")
    status = dev.steps(4, props)
    torch.cuda.synchronize()
    assert int(status.abs().max()) == 0
    for c in range(2):
        d = tmp_path / f"c{c}"
        d.mkdir()
        path = R.write_field(dev, str(d), props, column=c, ihist=4)
        cols, hdr = R.read_field(path, 1.0, props, ireset=0, idtold=1)
        assert hdr["m"] == 4
        ref = F.resume(F.parse(open(path).read()), 1.0, props, ireset=0, idtold=1)
        resumed = cols.to("cuda")
        for step in range(3):
            st = resumed.steps(1, props)
            torch.cuda.synchronize()
            assert int(st.abs().max()) == 0
            assert O.col_step(ref, n, 1.0, props) == 0
            host = resumed.to(None)
            for k, v in ref.items():
                assert np.array_equal(host.arrays[k][0], v), (c, step, k)


def test_checkpoint_continues_columns_bit_for_bit(tmp_path):
    """Device columns stepped, checkpointed from device memory, restored and stepped again
    equal the same columns stepped without a break, bit for bit (the whole state)."""
    import torch
    from lica_boiling1d_b200 import restart as R
    from lica_boiling1d_b200.column import ColumnProps, Columns
    props = ColumnProps(denr=1000.0, visr=20.0, tcr=25.0)
    n = 256
    a = Columns.film(n, 1.0, [0.08, 0.2], props).to("cuda")
    b = a.to("cuda")
    assert int(a.steps(3, props).abs().max()) == 0
    path = R.save_checkpoint(str(tmp_path / "c.npz"), a, props)
    restored, p2 = R.load_checkpoint(path)
    restored = restored.to("cuda")
    assert int(restored.steps(3, p2).abs().max()) == 0
    assert int(b.steps(6, props).abs().max()) == 0
    torch.cuda.synchronize()
    x, y = restored.to(None), b.to(None)
    for k in x.arrays:
        assert np.array_equal(x.arrays[k], y.arrays[k]), k


def test_checkpoint_continues_the_film_step(tmp_path):
    """The 2-D film: one step, a checkpoint, a fresh Film2D from it and one more step equal
    two steps without a break, bit for bit."""
    import torch
    from lica_boiling1d_b200 import film2d as G
    from lica_boiling1d_b200 import restart as R
    nx, ny = 64, 192
    P = G.default_props()
    st0 = G.initial_state(nx, ny, y0_cells=8, amp_cells=2, props=P)
    dt = G.stable_dt(nx, P)
    g1 = G.Film2D(nx, ny, P)
    cont = G.to_device(st0)
    g1.step(cont, dt)
    torch.cuda.synchronize()
    path = R.save_checkpoint(str(tmp_path / "f.npz"), cont, P)
    g1.step(cont, dt)
    torch.cuda.synchronize()
    g1.close()
    fields, P2 = R.load_checkpoint(path)
    g2 = G.Film2D(nx, ny, P2)
    dev = G.to_device(fields)
    g2.step(dev, dt)
    torch.cuda.synchronize()
    g2.close()
    a, b = G.to_host(dev), G.to_host(cont)
    for k in G.FIELDS:
        assert np.array_equal(a[k], b[k]), k
