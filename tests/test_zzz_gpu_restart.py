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
