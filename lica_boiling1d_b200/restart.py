"""Restart files of 1-D columns in the reference's ``fld######`` format (WRITEFIELD,
1d.f:1121-1232; PREFLD, 1d.f:972-1098), through the library's host-side reader and writer
(lica_col_fld_*).

``write_field`` writes one column of a ``Columns`` state (host or device) as the file the
reference writes every NPRINT steps; ``read_field`` reads such a file into a one-column
``Columns`` state that starts the time loop the way the reference does after IREAD = 1:
the band rebuilt from the lists, PSIF / PSI_CN / PSI_ZN recomputed, VOL_TOT_IPHS =
VOL_TOT_ORI and the step counter M back at 0.  The file keeps 13 significant digits
(ES20.12), so a resumed run continues from the written state rounded to that precision.

``save_checkpoint`` / ``load_checkpoint`` keep a complete state (columns, uneven column
batches, the 2-D film) bit for bit in a binary .npz, so that a run continues exactly.
"""
import ctypes as C
import os

import numpy as np

from . import native
from .column import Columns

# lica.in's switches and the reference's contact-state defaults (1d.f:573-582)
DEFAULT_OPTIONS = dict(ireset=1, idtold=0, ipzero=0)
DEFAULT_INFO = dict(ihist=0, qvol_ori=0.0, fk=0.0, ips=1, ipx=1, ipy=1, ipz=3, contact=0, contact_old=0,
                    contact_start=0.0, contact_time=0.0, lvson=1, t_con=100.0)


def field_name(ihist):
    """The reference's name for history record IHIST: "fld" and six digits."""
    buf = C.create_string_buffer(16)
    native.check(native.lib().lica_fld_name(int(ihist), buf, len(buf)), "lica_fld_name")
    return buf.value.decode()


def _host_column(cols, column):
    """Column `column` of a Columns or ColumnBatch state as host arrays, and its size n."""
    from .column import ColumnBatch
    if isinstance(cols, ColumnBatch):
        return {k: np.ascontiguousarray(v) for k, v in cols.column(column).items()}, int(cols.n[column])
    host = cols.to(None) if cols.on_device else cols
    return {k: np.ascontiguousarray(v[column]) for k, v in host.arrays.items()}, cols.n


def _state(arrays):
    return native.ColState(*[arrays[k].ctypes.data for k in native.COL_FIELDS])


def write_field(cols, path, props=None, *, column=0, **info):
    """Write column `column` of `cols` (a ``Columns`` or an uneven ``ColumnBatch``, host or
    device) to `path` (a directory gets the file name of ``info['ihist']``).  props: the
    column's properties (a batch's own by default).  info: ihist, qvol_ori, fk, ips, ipx,
    ipy, ipz and the contact state (DEFAULT_INFO).  Returns the path written."""
    unknown = set(info) - set(DEFAULT_INFO)
    if unknown:
        raise TypeError(f"unknown fld fields: {sorted(unknown)}")
    vals = dict(DEFAULT_INFO, **info)
    if os.path.isdir(path):
        path = os.path.join(path, field_name(vals["ihist"]))
    one, n = _host_column(cols, column)
    if props is None:
        if not hasattr(cols, "props"):
            raise TypeError("write_field: props is required for a Columns state")
        props = cols.props[column]
    fi = native.FldInfo(**vals)
    cp = props.c()
    native.check(native.lib().lica_col_fld_write(os.fsencode(path), n, C.byref(cp), C.byref(_state(one)),
                                                 C.byref(fi)), "lica_col_fld_write")
    return path


def field_size(path):
    """The column size n of a restart file."""
    n = C.c_int32()
    native.check(native.lib().lica_col_fld_dims(os.fsencode(path), C.byref(n)), "lica_col_fld_dims")
    return int(n.value)


def read_field(path, length, props, **options):
    """Read a restart file into a one-column host ``Columns`` of the column `length`.
    options: ireset, idtold, ipzero (DEFAULT_OPTIONS, lica.in's).  Returns (cols, header)
    with the file's header values as a dict."""
    unknown = set(options) - set(DEFAULT_OPTIONS)
    if unknown:
        raise TypeError(f"unknown options: {sorted(unknown)}")
    n = field_size(path)
    cols = Columns.empty(1, n, length)
    one = {k: np.ascontiguousarray(v[0]) for k, v in cols.arrays.items()}
    fi = native.FldInfo()
    opt = native.FldOptions(**dict(DEFAULT_OPTIONS, **options))
    cp = props.c()
    native.check(native.lib().lica_col_fld_read(os.fsencode(path), n, float(length), C.byref(cp), C.byref(opt),
                                                C.byref(_state(one)), C.byref(fi)), "lica_col_fld_read")
    for k in cols.arrays:
        cols.arrays[k][0] = one[k]
    header = {name: getattr(fi, name) for name, _ in native.FldInfo._fields_}
    return cols, header


# ------------------------------------------------------------------------------------
# Binary checkpoints: the complete state, bit for bit (the fld file keeps 13 digits and
# only the fields the reference writes).

CHECKPOINT_VERSION = 1


def _props_dict(p):
    from dataclasses import asdict
    return asdict(p)


def save_checkpoint(path, state, props=None):
    """Save a ``Columns``, a ``ColumnBatch`` (host or device) or a 2-D film state (the dict
    of Film2D's fields, host or device, with `props` its property dict) to `path` (.npz).
    Every array is saved exactly; resuming from it continues the run bit for bit."""
    import json

    from .column import ColumnBatch, Columns
    meta = dict(version=CHECKPOINT_VERSION)
    arrays = {}
    if isinstance(state, ColumnBatch):
        host = state.to(None) if not isinstance(state.arrays["w"], np.ndarray) else state
        meta.update(kind="column_batch", props=[_props_dict(p) for p in state.props])
        arrays.update({"a_" + k: v for k, v in host.arrays.items()})
        arrays.update(n=state.n, length=state.length)
    elif isinstance(state, Columns):
        if props is None:
            raise TypeError("save_checkpoint: props is required for a Columns state")
        host = state.to(None) if state.on_device else state
        meta.update(kind="columns", n=state.n, length=state.length, props=_props_dict(props))
        arrays.update({"a_" + k: v for k, v in host.arrays.items()})
    elif isinstance(state, dict) and set(state) >= {"u", "v", "p", "th", "phi"}:
        meta.update(kind="film2d", props=dict(props or {}))
        for k in ("u", "v", "p", "th", "phi"):
            v = state[k]
            arrays["a_" + k] = v if isinstance(v, np.ndarray) else v.detach().cpu().numpy()
    else:
        raise TypeError("save_checkpoint: a Columns, ColumnBatch or film state dict is expected")
    with open(path, "wb") as f:
        np.savez(f, meta=np.array(json.dumps(meta)), **arrays)
    return path


def load_checkpoint(path):
    """(state, props) saved by save_checkpoint, on the host: a ``Columns`` with its
    ColumnProps, a ``ColumnBatch`` (its props inside), or a film dict with its property
    dict."""
    import json

    from .column import ColumnBatch, ColumnProps, Columns
    with np.load(path, allow_pickle=False) as z:
        meta = json.loads(str(z["meta"]))
        if meta.get("version") != CHECKPOINT_VERSION:
            raise ValueError(f"{path}: checkpoint version {meta.get('version')} is not {CHECKPOINT_VERSION}")
        arrays = {k[2:]: z[k].copy() for k in z.files if k.startswith("a_")}
        kind = meta["kind"]
        if kind == "columns":
            return Columns(meta["n"], meta["length"], arrays), ColumnProps(**meta["props"])
        if kind == "column_batch":
            props = [ColumnProps(**p) for p in meta["props"]]
            b = ColumnBatch(z["n"].copy(), z["length"].copy(), props, arrays)
            return b, None
        if kind == "film2d":
            return arrays, meta["props"]
    raise ValueError(f"{path}: unknown checkpoint kind {kind!r}")


# ------------------------------------------------------------------------------------
# History records: WRITEHISTORY (1d.f:1235-1254), written every NPIN steps (1d.f:261-265)


def _fortran_es(x, w, d):
    x = float(x)
    if np.isnan(x):
        s = "NaN"
    elif np.isinf(x):
        s = ("-Infinity" if x < 0 else "Infinity") if w >= 9 else ("-Inf" if x < 0 else "Inf")
    else:
        m, e = ("%.*E" % (d, x)).split("E")
        e = int(e)
        s = m + ("E%+03d" % e if abs(e) <= 99 else "%+04d" % e)
    return s.rjust(w) if len(s) <= w else "*" * w


def _fortran_f(x, w, d):
    s = "%.*f" % (d, float(x))
    return s.rjust(w) if len(s) <= w else "*" * w


def history_record(cols, column=0):
    """The record WRITEHISTORY writes to fort.13 after a step, FORMAT(F13.5,4ES15.7):
    TIME, DT, CFLM (the step's CFL number), DVMAX (CONVRGE1's largest |div u - source|)
    and QMMAX, which the reference never assigns (written here as 0)."""
    from .column import ColumnBatch
    if isinstance(cols, ColumnBatch):
        one = cols.column(column)
        scal, stats = one["scal"], one["stats"]
    else:
        host = cols.to(None) if cols.on_device else cols
        scal, stats = host.arrays["scal"][column], host.arrays["stats"][column]
    return (_fortran_f(scal[1], 13, 5) + _fortran_es(scal[0], 15, 7) + _fortran_es(stats[0], 15, 7) +
            _fortran_es(stats[1], 15, 7) + _fortran_es(0.0, 15, 7) + "\n")
