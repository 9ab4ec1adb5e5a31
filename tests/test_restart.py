"""fld###### restart files of a 1-D column (lica_col_fld_*, host code): the writer's text
against the oracle's restatement of WRITEFIELD byte for byte, the reader's state against the
oracle's PREFLD + LVSINIT read branch + GRID_COUPLING(1) bit for bit, Fortran's edit
descriptor rules on output and input, the committed golden file, the reference's restart
semantics, and the error paths."""
import os

import numpy as np
import pytest

from oracle import fld as F
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fld_column_n16.txt")


def _props(**kw):
    from lica_boiling1d_b200.column import ColumnProps
    return ColumnProps(**kw)


def _cols(st, n, length=1.0):
    from lica_boiling1d_b200.column import Columns
    return Columns(n, length, {k: v[None].copy() for k, v in st.items()})


def _evolved(n, z0, steps, props, length=1.0):
    st = O.col_init(n, length, z0, props)
    for _ in range(steps):
        assert O.col_step(st, n, length, props) == 0
    return st


def test_es_and_i_edit_descriptors():
    """ES20.12 and I8 output: the known answers of the Fortran edit descriptors."""
    assert F.format_es(1.0) == "  1.000000000000E+00"
    assert F.format_es(-2.5e-3) == " -2.500000000000E-03"
    assert F.format_es(0.0) == "  0.000000000000E+00"
    assert F.format_es(-0.0) == " -0.000000000000E+00"
    assert F.format_es(123456789.0) == "  1.234567890000E+08"
    assert F.format_es(0.99999999999999) == "  1.000000000000E+00"
    assert F.format_es(1e-300) == "  1.000000000000-300"
    assert F.format_es(-1.5e200) == " -1.500000000000+200"
    assert F.format_es(float("nan")) == " " * 17 + "NaN"
    assert F.format_es(float("-inf")) == " " * 11 + "-Infinity"
    assert F.format_i(123) == "     123" and F.format_i(-7) == "      -7"
    assert F.format_i(123456789) == "********"


def test_library_formats_like_the_oracle(tmp_path):
    """Values of every exponent range, signed zeros and non-finite values through the
    library's writer: the W records equal the oracle's ES20.12 text."""
    from lica_boiling1d_b200 import restart as R
    n = 16
    props = _props()
    st = O.col_init(n, 1.0, 0.3, props)
    vals = [1.0, -2.5e-3, 0.0, -0.0, 1e-300, -1.5e200, 5e-324, 1.7976931348623157e308, 0.1, 1 / 3, -2 / 3,
            9.9999999999995e-5, 12345.678901234567, float("nan"), float("inf"), -1e100, 1e99]
    st["w"][1:1 + len(vals)] = vals
    path = R.write_field(_cols(st, n), str(tmp_path / "fldfmt"), props)
    assert open(path).read() == F.write_column(st, n, props, dict(R.DEFAULT_INFO))


@pytest.mark.parametrize("n,z0,steps", [(16, 0.3, 0), (32, 0.2, 5), (128, 0.1, 12), (256, 0.0607, 3)])
def test_writer_and_reader_match_the_oracle(tmp_path, n, z0, steps):
    from lica_boiling1d_b200 import restart as R
    props = _props()
    st = _evolved(n, z0, steps, props)
    info = dict(R.DEFAULT_INFO, ihist=steps + 1, qvol_ori=0.25, fk=-3.5, contact_time=1.5e-3)
    path = R.write_field(_cols(st, n), str(tmp_path), props, **info)
    assert os.path.basename(path) == "fld%06d" % (steps + 1)
    text = open(path).read()
    assert text == F.write_column(st, n, props, info)
    for opts in (dict(), dict(ireset=0, idtold=1), dict(ipzero=1)):
        cols, hdr = R.read_field(path, 1.0, props, **opts)
        ref = F.resume(F.parse(text), 1.0, props, **opts)
        for k, v in ref.items():
            assert np.array_equal(cols.arrays[k][0], v), (opts, k)
    assert hdr["ihist"] == steps + 1 and hdr["m"] == steps and hdr["n_max"] == 11
    assert hdr["qvol_ori"] == 0.25 and hdr["fk"] == -3.5 and hdr["t_con"] == 100.0 and hdr["lvson"] == 1


def test_round_trip_keeps_thirteen_digits(tmp_path):
    """read(write(state)): the written fields to ES20.12's 13 significant digits, the band
    exactly, PSIF and the coupled fractions recomputed from the rounded band."""
    from lica_boiling1d_b200 import restart as R
    n, props = 128, _props()
    st = _evolved(n, 0.1, 10, props)
    path = R.write_field(_cols(st, n), str(tmp_path), props, ihist=10)
    cols, _ = R.read_field(path, 1.0, props, ireset=0, idtold=1)
    got = {k: v[0] for k, v in cols.arrays.items()}
    for k, sl in (("w", slice(1, n + 2)), ("p", slice(1, n + 1)), ("t", slice(0, n + 2))):
        np.testing.assert_allclose(got[k][sl], st[k][sl], rtol=5e-13, atol=1e-300)
    assert np.array_equal(got["layer"], st["layer"])
    band = st["layer"] > 0
    np.testing.assert_allclose(got["phi"][band], st["phi"][band], rtol=5e-13, atol=1e-300)
    assert np.abs(got["psif"] - st["psif"]).max() < 1e-12
    assert np.abs(got["psi_cn"] - st["psi_cn"]).max() < 1e-12
    assert got["scal"][2] == 0.0
    np.testing.assert_allclose(got["scal"][[0, 1, 3, 4]], st["scal"][[0, 1, 3, 3]], rtol=5e-13)


def test_resumed_run_continues_the_physics(tmp_path):
    """The reference's restart semantics: the file holds no MFLVS / IMASK and the step
    counter starts again at 1, so the first resumed step moves no interface (no interfacial
    mass flux yet); from then on the resumed column follows the continuous one a step
    behind: its height after step i+1 is the continuous height after step i to within a
    hundredth of a step's growth, and the temperatures agree to 1e-8."""
    from lica_boiling1d_b200 import restart as R
    n, props = 128, _props()
    st = _evolved(n, 0.1, 20, props)
    path = R.write_field(_cols(st, n), str(tmp_path), props, ihist=1)
    cols, _ = R.read_field(path, 1.0, props, ireset=0, idtold=1)
    rs = {k: v[0].copy() for k, v in cols.arrays.items()}
    h_start = st["stats"][5]
    hs, hr = [], []
    for _ in range(7):
        assert O.col_step(st, n, 1.0, props) == 0 and O.col_step(rs, n, 1.0, props) == 0
        hs.append(st["stats"][5])
        hr.append(rs["stats"][5])
        assert np.abs(st["t"] - rs["t"]).max() < 1e-8
    assert abs(hr[0] - h_start) < 0.01 * (hs[0] - h_start)
    for i in range(6):
        growth = hs[i + 1] - hs[i]
        assert growth > 0 and abs(hr[i + 1] - hs[i]) < 0.01 * growth


def _write_golden_case():
    props = _props()
    st = _evolved(16, 0.3, 2, props)
    return st, props


def test_golden_file(tmp_path):
    """The committed file (tests/golden/make_fld_fixture.py): the library writes it byte for
    byte from the same state and reads it to the oracle's resumed state."""
    from lica_boiling1d_b200 import restart as R
    st, props = _write_golden_case()
    gold = open(GOLDEN).read()
    path = R.write_field(_cols(st, 16), str(tmp_path / "g"), props, ihist=2)
    assert open(path).read() == gold
    cols, hdr = R.read_field(GOLDEN, 1.0, props)
    ref = F.resume(F.parse(gold), 1.0, props)
    for k, v in ref.items():
        assert np.array_equal(cols.arrays[k][0], v), k
    assert hdr["ihist"] == 2 and hdr["m"] == 2


def _edit(text, line_no, new):
    lines = text.split("\n")
    lines[line_no] = new
    return "\n".join(lines)


def test_fortran_input_forms(tmp_path):
    """PREFLD's formatted input: D exponents, exponents without a letter, fields without a
    decimal point (the last 12 digits are the fraction), blank fields (zero) and records
    shorter than their fields; the library and the oracle read them alike."""
    from lica_boiling1d_b200 import restart as R
    n, props = 16, _props()
    st = O.col_init(n, 1.0, 0.3, props)
    text = F.write_column(st, n, props, dict(R.DEFAULT_INFO))
    lines = text.split("\n")
    # locate the P record: after the header (4), U, V and W records
    N3 = n + 1
    nu, nv, nw = 2 * 3 * (N3 + 1), 3 * 2 * (N3 + 1), 9 * N3
    p0 = 4 + -(-nu // 5) + -(-nv // 5) + -(-nw // 5)
    fields = ["  1.5D+00", "    25-1", "1234567890123", "", "-7.25e+3"]
    lines[p0] = "".join(f.rjust(20) for f in fields[:-1])[:61]   # short record: 4th field blank, 5th missing
    lines[p0] += fields[3].rjust(19)
    lines[p0 + 1] = "".join(["-7.25e+3".rjust(20)] * 5)
    edited = "\n".join(lines)
    path = tmp_path / "fld000000"
    path.write_text(edited)
    cols, _ = R.read_field(str(path), 1.0, props)
    ref = F.resume(F.parse(edited), 1.0, props)
    p = cols.arrays["p"][0]
    assert np.array_equal(p, ref["p"])
    assert p[1] == 1.5 and p[2] == 25e-13 and p[3] == 1.234567890123 and p[4] == 0.0 and p[5] == 0.0
    assert p[6] == -7250.0


def test_columns_of_an_uneven_batch(tmp_path):
    """Each column of an uneven batch (its own size and properties) written from the batch
    equals the oracle's WRITEFIELD of that column's state."""
    from lica_boiling1d_b200 import restart as R
    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    n, length, z0, props = uneven_batch(4, seed=3, nmin=16, nmax=96)
    b = ColumnBatch.films(n, length, z0, props)
    for c in range(4):
        d = tmp_path / f"c{c}"
        d.mkdir()
        path = R.write_field(b, str(d), column=c, ihist=c)
        st = b.column(c)
        assert open(path).read() == F.write_column(st, int(n[c]), props[c], dict(R.DEFAULT_INFO, ihist=c))
        cols, _ = R.read_field(path, float(length[c]), props[c])
        assert cols.n == int(n[c]) and np.array_equal(cols.arrays["layer"][0], st["layer"])


def test_binary_checkpoints_are_exact(tmp_path):
    """save_checkpoint / load_checkpoint keep every array of a column state, an uneven batch
    and a 2-D film state bit for bit, and a column resumed from one continues exactly."""
    from lica_boiling1d_b200 import film2d
    from lica_boiling1d_b200 import restart as R
    from lica_boiling1d_b200.column import ColumnBatch, uneven_batch
    n, props = 64, _props(denr=800.0, jakob=0.02)
    st = _evolved(n, 0.15, 6, props)
    path = R.save_checkpoint(str(tmp_path / "c.npz"), _cols(st, n), props)
    cols, p2 = R.load_checkpoint(path)
    assert p2 == props and cols.n == n and cols.length == 1.0
    for k, v in st.items():
        a = cols.arrays[k][0]
        assert a.dtype == v.dtype and np.array_equal(a, v), k
    resumed = {k: v[0].copy() for k, v in cols.arrays.items()}
    for _ in range(3):
        assert O.col_step(st, n, 1.0, props) == 0 and O.col_step(resumed, n, 1.0, p2) == 0
    for k, v in st.items():
        assert np.array_equal(resumed[k], v), k

    nb, length, z0, bprops = uneven_batch(3, seed=5, nmin=16, nmax=80)
    b = ColumnBatch.films(nb, length, z0, bprops)
    path = R.save_checkpoint(str(tmp_path / "b.npz"), b)
    b2, _ = R.load_checkpoint(path)
    assert np.array_equal(b2.n, b.n) and np.array_equal(b2.length, b.length) and b2.props == b.props
    assert np.array_equal(b2.offsets, b.offsets)
    for k, v in b.arrays.items():
        assert np.array_equal(b2.arrays[k], v), k

    fp = film2d.default_props()
    fs = film2d.initial_state(64, 96, 24.0, 2.0, fp)
    path = R.save_checkpoint(str(tmp_path / "f.npz"), fs, fp)
    f2, fp2 = R.load_checkpoint(path)
    assert fp2 == fp
    for k in film2d.FIELDS:
        assert np.array_equal(f2[k], fs[k]), k
    with pytest.raises(TypeError):
        R.save_checkpoint(str(tmp_path / "x.npz"), {"w": 1})


def test_history_record():
    """WRITEHISTORY's record (FORMAT(F13.5,4ES15.7)) of the column's last step."""
    from lica_boiling1d_b200 import restart as R
    n, props = 64, _props()
    st = _evolved(n, 0.1, 3, props)
    rec = R.history_record(_cols(st, n))
    assert len(rec) == 13 + 4 * 15 + 1 and rec.endswith("\n")
    f = [rec[:13]] + [rec[13 + 15 * q:28 + 15 * q] for q in range(4)]
    assert f[0] == "%13.5f" % st["scal"][1]
    assert float(f[1]) == float("%.7E" % st["scal"][0]) and float(f[2]) == float("%.7E" % st["stats"][0])
    assert float(f[3]) == float("%.7E" % st["stats"][1]) and f[4] == "  0.0000000E+00"


def test_field_names():
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200 import restart as R
    assert R.field_name(0) == "fld000000"
    assert R.field_name(42) == "fld000042"
    assert R.field_name(999999) == "fld999999"
    for bad in (-1, 1000000):
        with pytest.raises(native.LicaError):
            R.field_name(bad)


def test_errors(tmp_path):
    from lica_boiling1d_b200 import native
    from lica_boiling1d_b200 import restart as R
    n, props = 16, _props()
    st = O.col_init(n, 1.0, 0.3, props)
    text = F.write_column(st, n, props, dict(R.DEFAULT_INFO))

    def read(t):
        p = tmp_path / "f"
        p.write_text(t)
        return R.read_field(str(p), 1.0, props)

    with pytest.raises(native.LicaError, match="LICA_ERR_IO"):
        R.read_field(str(tmp_path / "missing"), 1.0, props)
    with pytest.raises(native.LicaError, match="LICA_ERR_IO"):
        read("\n".join(text.split("\n")[:40]))                       # truncated
    with pytest.raises(native.LicaError, match="LICA_BAD_ARG"):
        read(_edit(text, 0, "       3       2      17"))              # not a column
    with pytest.raises(native.LicaError, match="LICA_ERR_IO"):
        read(_edit(text, 1, "       0       0  1.0000000x0000E+00  2.500000000000E-06"))   # bad field
    lines = text.split("\n")
    i1013 = next(i for i, ln in enumerate(lines) if ln == "       1      11")
    with pytest.raises(native.LicaError, match="LICA_BAD_ARG"):
        read(_edit(text, i1013, "       2      11"))                   # two level sets
    band0 = i1013 + 4
    k = int(lines[band0][16:24])
    with pytest.raises(native.LicaError, match="LICA_BAD_ARG"):
        read(_edit(text, band0, lines[band0][:16] + "%8d" % (2 * n + 9) + lines[band0][24:]))   # K outside
    with pytest.raises(native.LicaError, match="LICA_BAD_ARG"):
        read(_edit(text, band0, "       3" + lines[band0][8:]))          # I outside 1..2
    assert k > 1
    with pytest.raises(native.LicaError, match="LICA_BAD_ARG"):
        R.write_field(_cols(st, n), str(tmp_path), props, ihist=10 ** 6)
