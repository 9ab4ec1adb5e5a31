"""Writes tests/golden/column_oracle_n64.npz: the oracle's complete column state (oracle/
column1d.cpp) after 0, 3 and 6 time steps for two 64-cell columns -- the shipped lica.in
properties with a film 0.1 thick, and density ratio 800, Jakob 0.02 with a film 0.3 thick.
It pins the oracle's uniform-grid arithmetic bit for bit, so a refactor of the oracle (such
as per-cell metrics) is checked against it.  Run from the repository root:
python tests/golden/make_column_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lica_boiling1d_b200.column import ColumnProps  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [("ship", 0.1, {}), ("dense", 0.3, dict(denr=800.0, jakob=0.02))]
N = 64


def trajectory(z0, kw):
    props = ColumnProps(**kw)
    st = O.col_init(N, 1.0, z0, props)
    out = {}
    for step in range(7):
        if step in (0, 3, 6):
            out.update({f"s{step}_{k}": v.copy() for k, v in st.items()})
        if step < 6:
            assert O.col_step(st, N, 1.0, props) == 0
    return out


if __name__ == "__main__":
    arrays = {}
    for name, z0, kw in CASES:
        arrays.update({f"{name}_{k}": v for k, v in trajectory(z0, kw).items()})
    np.savez_compressed(os.path.join(HERE, "column_oracle_n64.npz"), **arrays)
