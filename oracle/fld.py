"""ORACLE (test infrastructure only): the reference's fld###### restart file of a 1-D column.

A Python restatement of WRITEFIELD (1d.f:1121-1232) and PREFLD (1d.f:972-1098) -- the
records and their FORMATs 1001-1016 -- with Fortran's formatted output and input rules for
the ES and I edit descriptors (Fortran 2008 10.7.2), and of the start-up that follows a read
in MAIN (LVSINIT's read branch, two_phase.f:148-205, and GRID_COUPLING(1), through
orc_col_resume in column1d.cpp; VOL_TOT_IPHS = VOL_TOT_ORI, 1d.f:146-151; IRESET,
1d.f:175-178; IDTOLD, 1d.f:1080-1085; IPZERO, 1d.f:1055).

Parity of the text itself is pinned to the FORMAT statements and the language's edit
descriptors only: the reference ships no fld file (lica.in names fld100000, not included)
and no Fortran compiler is available to run WRITEFIELD.

The 1-D column is the reference's grid.in case N1 = N2 = 2, N3 = n + 1, N1F = N2F = 3,
N3F = 2n + 1; fields are repeated over their (I, J) replicas and read from I = J = 1.
"""
import math

import numpy as np

M_MAX = 11

# FORMAT statements of WRITEFIELD / PREFLD: one record's descriptors, (kind, w, d)
I8 = ("I", 8, 0)
ES = ("ES", 20, 12)
FORMATS = {
    1001: [I8] * 3, 1002: [I8, I8, ES, ES], 1003: [I8] * 4 + [ES], 1004: [ES], 1005: [ES] * 5, 1006: [ES] * 3,
    1007: [I8] * 4, 1011: [I8] * 3, 1012: [ES] * 6, 1013: [I8] * 2, 1014: [ES] * 8, 1015: [I8] * 8,
    1016: [I8, I8, I8, ES],
}


def format_es(x, w=20, d=12):
    """ESw.d output: x = m 10^e with 1 <= |m| < 10 rounded to d decimals; exponent E+zz for
    |e| <= 99, +zzz for larger; right-justified; w asterisks when it does not fit."""
    x = float(x)
    if math.isnan(x):
        s = "NaN"
    elif math.isinf(x):
        s = ("-Infinity" if x < 0 else "Infinity") if w >= 9 else ("-Inf" if x < 0 else "Inf")
    else:
        m, e = ("%.*E" % (d, x)).split("E")
        e = int(e)
        s = m + ("E%+03d" % e if abs(e) <= 99 else "%+04d" % e)
    return s.rjust(w) if len(s) <= w else "*" * w


def format_i(v, w=8):
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def _put(fmt, items):
    """One WRITE statement: records of len(fmt) items (format reversion); an empty list
    still writes one record."""
    out = []
    per = len(FORMATS[fmt])
    desc = FORMATS[fmt]
    if not items:
        return "\n"
    for i in range(0, len(items), per):
        rec = items[i:i + per]
        out.append("".join(format_i(v) if desc[q][0] == "I" else format_es(v) for q, v in enumerate(rec)) + "\n")
    return "".join(out)


def band_lists(layer, n):
    """NUMA and the (I, J, K) lists of a column: per layer the cells in ascending K, each on
    its four refined (I, J) replicas."""
    nf = 2 * n
    lists = {m: [] for m in range(1, M_MAX + 1)}
    for k in range(-2, nf + 5):
        m = int(layer[k + 2])
        if m:
            lists[m].append(k)
    return lists


def write_column(st, n, props, info):
    """The text WRITEFIELD writes for one column state (dict of the column arrays).  info:
    ihist, qvol_ori, fk, ips, ipx, ipy, ipz and the contact state."""
    N1, N2, N3 = 2, 2, n + 1
    w, p, t, phi, layer, scal = st["w"], st["p"], st["t"], st["phi"], st["layer"], st["scal"]
    o = [_put(1001, [N1, N2, N3]), _put(1002, [info["ihist"], int(scal[2]), scal[1], scal[0]]),
         _put(1003, [info["ips"], info["ipx"], info["ipy"], info["ipz"], props.prm]), _put(1004, [info["qvol_ori"]])]
    o.append(_put(1005, [0.0] * (N1 * (N2 + 1) * (N3 + 1))))
    o.append(_put(1005, [0.0] * ((N1 + 1) * N2 * (N3 + 1))))
    o.append(_put(1005, [w[k] for k in range(1, N3 + 1) for _j in range(N2 + 1) for _i in range(N1 + 1)]))
    o.append(_put(1005, [p[k] for k in range(1, n + 1)]))
    o.append(_put(1011, [3, 3, 2 * n + 1]))
    o.append(_put(1012, [props.denr, props.visr, props.fr, props.weber, info["fk"], props.re]))
    o.append(_put(1013, [1, M_MAX]))
    o.append(_put(1014, [scal[3]]))
    lists = band_lists(layer, n)
    o.append(_put(1015, [4 * len(lists[m]) for m in range(1, M_MAX + 1)]))
    for m in range(1, M_MAX + 1):
        for k in lists[m]:
            for j in (1, 2):
                for i in (1, 2):
                    o.append(_put(1016, [i, j, k, phi[k + 2]]))
    o.append(_put(1007, [info["contact"]]))
    o.append(_put(1007, [info["contact_old"]]))
    o.append(_put(1005, [info["contact_start"]]))
    o.append(_put(1005, [info["contact_time"]]))
    o.append(_put(1007, [info["lvson"]]))
    o.append(_put(1005, [info["t_con"]]))
    if info["ips"] == 1:
        o.append(_put(1006, [props.prm, props.scr, props.tcr]))
        o.append(_put(1005, [t[k] for k in range(0, N3 + 1) for _j in range(N2 + 1) for _i in range(N1 + 1)]))
    return "".join(o)


def parse_int(f):
    """Iw input: blanks ignored (BLANK = 'NULL'); all blank reads 0."""
    s = f.replace(" ", "").replace("\t", "")
    if not s:
        return 0
    if s[0] in "+-":
        if len(s) == 1 or not s[1:].isdigit():
            raise ValueError(f"bad integer field {f!r}")
    elif not s.isdigit():
        raise ValueError(f"bad integer field {f!r}")
    return int(s)


def parse_real(f, d):
    """Ew.d / ESw.d input: [sign] digits [. digits] [exponent]; the exponent E|D|Q [sign]
    digits, or sign digits; without a decimal point the last d digits are the fraction;
    blanks ignored; NaN, Inf, Infinity."""
    s = f.replace(" ", "").replace("\t", "")
    if not s:
        return 0.0
    sign = ""
    if s[0] in "+-":
        sign, s = ("-" if s[0] == "-" else ""), s[1:]
    u = s.upper()
    if u in ("INF", "INFINITY"):
        return -math.inf if sign else math.inf
    if u.startswith("NAN") and (len(u) == 3 or (u[3] == "(" and u.endswith(")"))):
        return math.nan
    i = 0
    digits, point = "", None
    while i < len(s) and (s[i].isdigit() or s[i] == "."):
        if s[i] == ".":
            if point is not None:
                raise ValueError(f"bad real field {f!r}")
            point = len(digits)
        else:
            digits += s[i]
        i += 1
    if not digits:
        raise ValueError(f"bad real field {f!r}")
    ex = 0
    if i < len(s):
        if s[i].upper() in "EDQ":
            i += 1
        elif s[i] not in "+-":
            raise ValueError(f"bad real field {f!r}")
        rest = s[i:]
        if rest[:1] in ("+", "-"):
            esign, rest = rest[0], rest[1:]
        else:
            esign = "+"
        if not rest.isdigit():
            raise ValueError(f"bad real field {f!r}")
        ex = int(esign + rest)
    frac = d if point is None else len(digits) - point
    v = float(f"{sign}{digits}E{ex - frac}")
    if math.isinf(v):
        raise ValueError(f"real field {f!r} overflows")
    return v


class _Records:
    def __init__(self, text):
        self.lines = [ln[:-1] if ln.endswith("\r") else ln for ln in text.split("\n")]
        if text.endswith("\n"):
            self.lines.pop()
        self.next = 0

    def read(self, fmt, count):
        """One READ statement of count items under FORMAT fmt."""
        desc = FORMATS[fmt]
        out = []
        while True:
            if self.next >= len(self.lines):
                raise EOFError(f"end of file in FORMAT {fmt}")
            rec = self.lines[self.next]
            self.next += 1
            col = 0
            for kind, w, d in desc:
                if len(out) == count:
                    break
                f = rec[col:col + w]
                col += w
                out.append(parse_int(f) if kind == "I" else parse_real(f, d))
            if len(out) >= count:
                return out


def parse(text):
    """PREFLD's records of a column file: the header values and the raw arrays."""
    R = _Records(text)
    N1, N2, N3 = R.read(1001, 3)
    if (N1, N2) != (2, 2):
        raise ValueError(f"not a column: N1, N2 = {N1}, {N2}")
    r = dict(N1=N1, N2=N2, N3=N3)
    r["ihist"], r["m"], r["time"], r["dt"] = R.read(1002, 4)
    r["ips"], r["ipx"], r["ipy"], r["ipz"], r["pra"] = R.read(1003, 5)
    r["qvol_ori"], = R.read(1004, 1)
    r["U"] = R.read(1005, N1 * (N2 + 1) * (N3 + 1))
    r["V"] = R.read(1005, (N1 + 1) * N2 * (N3 + 1))
    r["W"] = np.array(R.read(1005, (N1 + 1) * (N2 + 1) * N3)).reshape(N3, N2 + 1, N1 + 1)   # [K-1, J, I]
    r["P"] = np.array(R.read(1005, (N3 - 1)))
    r["N1F"], r["N2F"], r["N3F"] = R.read(1011, 3)
    r["denr"], r["visr"], r["fr"], r["surf_j"], r["fk"], r["re_air"] = R.read(1012, 6)
    nlvs, nmax = R.read(1013, 2)
    if nlvs != 1 or not 0 <= nmax <= M_MAX:
        raise ValueError(f"NLVS, N_MAX = {nlvs}, {nmax}")
    r["n_max"] = nmax
    r["vol_tot_ori"], = R.read(1014, 1)
    r["numa"] = R.read(1015, nmax)
    r["band"] = [[tuple(R.read(1016, 4)) for _ in range(r["numa"][m])] for m in range(nmax)]
    r["contact"], = R.read(1007, 1)
    r["contact_old"], = R.read(1007, 1)
    r["contact_start"], = R.read(1005, 1)
    r["contact_time"], = R.read(1005, 1)
    r["lvson"], = R.read(1007, 1)
    r["t_con"], = R.read(1005, 1)
    r["T"] = None
    if r["ips"] == 1:
        r["prm"], r["scr"], r["tcr"] = R.read(1006, 3)
        r["T"] = np.array(R.read(1005, (N1 + 1) * (N2 + 1) * (N3 + 1))).reshape(N3 + 1, N2 + 1, N1 + 1)
    return r


def resume(r, length, props, *, ireset=1, idtold=0, ipzero=0):
    """The column state at the start of the time loop after reading r (parse()).  Returns a
    dict of the column arrays (the layout of oracle.col_empty)."""
    from . import oracle as O
    n = r["N3"] - 1
    nf = 2 * n
    st = O.col_empty(n)
    st["w"][1:n + 2] = r["W"][:, 1, 1]
    st["p"][1:n + 1] = r["P"]
    if ipzero == 1:
        st["p"][:] = 0.0
    if r["T"] is not None:
        st["t"][:] = r["T"][:, 1, 1]
    for m, cells in enumerate(r["band"], start=1):
        for i, j, k, a in cells:
            if not (1 <= i <= 2 and 1 <= j <= 2 and -2 <= k <= nf + 4):
                raise ValueError(f"band cell {(i, j, k)} outside the column")
            st["layer"][k + 2] = m
            if (i, j) == (1, 1):
                st["phi"][k + 2] = a
    L = O.lib()
    L.orc_col_resume(n, float(length), O._p(st["phi"]), O._pi(st["layer"]), O._p(st["psif"]), O._p(st["psi_cn"]),
                     O._p(st["psi_zn"]))
    st["scal"][:] = [r["dt"] if idtold == 1 else props.dt0, 0.0 if ireset == 1 else r["time"], 0.0,
                     r["vol_tot_ori"], r["vol_tot_ori"]]
    return st
