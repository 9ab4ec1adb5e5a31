"""Writes tests/golden/fld_column_n16.txt: the oracle's WRITEFIELD text (oracle/fld.py) for a
16-cell column (film 0.3 thick, the shipped lica.in properties) after two oracle time steps,
IHIST = 2.  Run from the repository root: python tests/golden/make_fld_fixture.py"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lica_boiling1d_b200.column import ColumnProps  # noqa: E402
from oracle import fld as F  # noqa: E402
from oracle import oracle as O  # noqa: E402

INFO = dict(ihist=2, qvol_ori=0.0, fk=0.0, ips=1, ipx=1, ipy=1, ipz=3, contact=0, contact_old=0, contact_start=0.0,
            contact_time=0.0, lvson=1, t_con=100.0)

if __name__ == "__main__":
    props = ColumnProps()
    st = O.col_init(16, 1.0, 0.3, props)
    for _ in range(2):
        assert O.col_step(st, 16, 1.0, props) == 0
    with open(os.path.join(HERE, "fld_column_n16.txt"), "w") as f:
        f.write(F.write_column(st, 16, props, INFO))
