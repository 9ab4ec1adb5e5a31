"""ORACLE (test infrastructure only): non-uniform grids.

A Python restatement of the reference's grid generator sections -- UNIFORM
(grid.f:326-345), GEOPRO (grid.f:348-380), HYPTAN (grid.f:383-420), dispatched by IOPT as
grid.f:118-128 does -- and of GEOMETRIC (1d.f:4808-4882) for one wall-bounded direction,
in double precision (the solver is built with -fdefault-real-8), with the C library's
tanh and pow through the math module.  Also the stretched wall-normal pressure operator:
POISSON's AK / CK = VVDZ SSDZ DENF_ZI (1d.f:3535-3541) in 2-D with x uniform and periodic,
both assembled directly (a sparse matrix, the known answer) and rescaled row by row into
the uniform multigrid's arrays.  And GEOM_COUPLING's z tables (1d.f:5037-5370) between a
flow grid of any spacing and the uniform level-set grid, with INTER_PSI's box mean over
general refined faces.

Parity with grid.f is pinned by the generator's formulas and known answers (end points,
progression ratios, symmetry); grid.f itself was not run (no Fortran compiler).
"""
import math

import numpy as np


def section(iopt, xyzi, xyzf, ngi, ngf, fac1, fac2, out):
    """Fill out[N - 1] for N = ngi..ngf."""
    if iopt == 1:
        dc = (xyzf - xyzi) / (ngf - ngi)
        for n in range(ngi, ngf + 1):
            out[n - 1] = xyzi + (n - ngi) * dc
    elif iopt == 2:
        er = float(fac1)
        if er == 1.0:
            raise ValueError("Expansion Ratio is 1")
        if fac2 != 1.0:
            er = 1.0 / er
        dsi = (xyzf - xyzi) * (1.0 - er) / (1.0 - er ** (ngf - ngi))
        for n in range(ngi + 1, ngf):
            out[n - 1] = xyzi + dsi * (1.0 - er ** (n - ngi)) / (1.0 - er)
        out[ngi - 1] = xyzi
        out[ngf - 1] = xyzf
    else:
        gam = float(fac1)
        if fac2 != 0.0:
            xsi = float(fac2)
            for n in range(ngi, ngf + 1):
                seg = float(n - ngi) / float(ngf - ngi)
                out[n - 1] = xyzi + (xyzf - xyzi) * xsi * (1.0 - math.tanh(gam * (xsi - seg)) / math.tanh(gam * xsi))
        else:
            xsi = 1.0
            for n in range(ngi, ngf + 1):
                seg = float(n - ngi) / float(ngf - ngi)
                out[n - 1] = xyzi + (xyzf - xyzi) * xsi * math.tanh(gam * seg) / math.tanh(gam * xsi)
    return out


def metrics(z):
    """GEOMETRIC for the faces z[0..n-1] = Z(1..n): SDZ, VDZ, SSDZ, VVDZ, ZP indexed 0..n."""
    n = len(z)
    Z = [0.0] + [float(v) for v in z]
    nm = n - 1
    sdz, vdz, ssdz, vvdz, zp = (np.zeros(n + 1) for _ in range(5))
    if nm == 1:
        sdz[1] = 1.0 / nm
        ssdz[1] = 1.0 / sdz[1]
        vdz[1] = sdz[1]
        vvdz[1] = ssdz[1]
    else:
        for k in range(1, nm + 1):
            sdz[k] = Z[k + 1] - Z[k]
        for k in range(2, nm + 1):
            vdz[k] = 0.5 * (sdz[k] + sdz[k - 1])
        vdz[1] = 0.5 * sdz[1]
        vdz[n] = 0.5 * sdz[nm]
        for k in range(1, nm + 1):
            ssdz[k] = 1.0 / sdz[k]
        for k in range(1, n + 1):
            vvdz[k] = 1.0 / vdz[k]
    for k in range(1, nm + 1):
        zp[k] = Z[k] + 0.5 * sdz[k]
    zp[n] = Z[n]
    zp[0] = Z[1]
    return dict(sdz=sdz, vdz=vdz, ssdz=ssdz, vvdz=vvdz, zp=zp)


def stretched_system(yface, bx, by, f):
    """The stretched system rescaled by each row's height for the multigrid with hy = 1."""
    ny, nx = f.shape
    y = np.asarray(yface, dtype=np.float64)
    bxo = np.empty((ny, nx))
    fo = np.empty((ny, nx))
    byo = np.empty((ny + 1, nx))
    for j in range(ny):
        dy = y[j + 1] - y[j]
        bxo[j] = bx[j] * dy
        fo[j] = f[j] * dy
    byo[0] = by[0]
    for j in range(1, ny + 1):
        dyb = y[j] - y[j - 1]
        vd = 0.5 * ((y[j + 1] - y[j]) + dyb) if j < ny else dyb
        byo[j] = by[j] / vd
    return bxo, byo, fo


def stretched_operator(yface, bx, by, hx):
    """The stretched operator itself (scipy CSR, rows j * nx + i): x periodic with spacing
    hx, y faces yface, Neumann bottom, p = 0 on the top face."""
    import scipy.sparse as sp
    ny, nx = bx.shape
    y = np.asarray(yface, dtype=np.float64)
    dy = np.diff(y)
    rows, cols, vals = [], [], []
    cx = 1.0 / (hx * hx)
    for j in range(ny):
        for i in range(nx):
            r = j * nx + i
            diag = 0.0
            for ii, b in (((i - 1) % nx, bx[j, i]), ((i + 1) % nx, bx[j, (i + 1) % nx])):
                rows.append(r)
                cols.append(j * nx + ii)
                vals.append(cx * b)
                diag -= cx * b
            if j > 0:
                a = by[j, i] / (0.5 * (dy[j] + dy[j - 1])) / dy[j]
                rows.append(r)
                cols.append((j - 1) * nx + i)
                vals.append(a)
                diag -= a
            if j < ny - 1:
                a = by[j + 1, i] / (0.5 * (dy[j + 1] + dy[j])) / dy[j]
                rows.append(r)
                cols.append((j + 1) * nx + i)
                vals.append(a)
                diag -= a
            else:
                diag -= by[ny, i] / (0.5 * dy[j]) / dy[j]
            rows.append(r)
            cols.append(r)
            vals.append(diag)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))


def coupling_z(z, zf):
    """GEOM_COUPLING's z tables (1d.f:5142-5190, 5308-5363) for flow faces z[0..n3-1] =
    Z(1..N3) and refined faces zf[0..n3f-1] = ZF(1..N3F); the same layout as the library's."""
    Z = [0.0] + [float(v) for v in z]
    ZF = [0.0] + [float(v) for v in zf]
    n3, n3f = len(Z) - 1, len(ZF) - 1
    n3m = n3 - 1
    ZP = [0.0] * (n3 + 1)
    for k in range(1, n3m + 1):
        ZP[k] = Z[k] + 0.5 * (Z[k + 1] - Z[k])
    ZP[n3] = Z[n3]
    ZP[0] = Z[1]
    sdzf = ZF[2] - ZF[1]
    ZPF = [0.0] + [ZF[k] + 0.5 * sdzf for k in range(1, n3f + 1)]

    def centre_below(zz):
        for kk in range(1, n3m + 1):
            if abs(zz - ZP[kk]) <= 1e-10:
                return kk
            if ZP[1] > zz:
                return 1
            if ZP[kk] > zz:
                return kk - 1
            if ZP[n3m] < zz:
                return n3m
        raise ValueError("Z-DIR FLOW_SOLVER->REFINED COUPLING PROBLEM")

    def pair(x):
        for kf in range(1, n3f + 1):
            if abs(ZF[kf] - x) <= 1e-10:
                return kf - 1, kf
            if ZF[kf] > x:
                return kf - 1, kf - 1
        raise ValueError("CAL KCOU HAVE PROBLEM")

    kv = np.zeros(n3f + 1, np.int32)
    kmv = np.zeros(n3f + 1, np.int32)
    for k in range(1, n3f + 1):
        kv[k] = centre_below(ZF[k])
        kmv[k] = centre_below(ZPF[k])
    K1, K2 = {}, {}
    for k in range(1, n3 + 1):
        K1[k], K2[k] = pair(Z[k])
    for T in (K1, K2):
        T[0] = T[1] - (T[n3m] - T[n3m - 1])
        T[-1] = T[0] - (T[n3m - 1] - T[n3m - 2])
        T[n3 + 1] = T[n3] + (T[2] - T[1])
        T[n3 + 2] = T[n3 + 1] + (T[3] - T[2])
    M1, M2 = {}, {}
    for k in range(1, n3m + 1):
        M1[k], M2[k] = pair(ZP[k])
    for T in (M1, M2):
        T[0] = T[1] - (T[n3m] - T[n3m - 1])
        T[-1] = T[0] - (T[n3m - 1] - T[n3m - 2])
        T[n3] = T[n3m] + (T[n3m] - T[n3m - 1])
        T[n3 + 1] = T[n3] + (T[2] - T[1])
    return dict(kcou1=np.array([K1[k] for k in range(-1, n3 + 3)], np.int32),
                kcou2=np.array([K2[k] for k in range(-1, n3 + 3)], np.int32),
                kcoump1=np.array([M1[k] for k in range(-1, n3 + 2)], np.int32),
                kcoump2=np.array([M2[k] for k in range(-1, n3 + 2)], np.int32), kcou_vel=kv, kcoump_vel=kmv)


def box_mean(f, zf, k1, k2, z1, z2):
    """The z part of INTER_PSI (two_phase.f:5123-5538) over [z1, z2] and refined cells
    k1..k2 with refined faces zf (zf[k - 1] = ZF(k)) and values f[k] (k = 1..n3f-1): the
    overlap-weighted mean, by the reference's case analysis, once per (II, JJ) replica."""
    nf = len(zf) - 1
    ssdzf = 1.0 / (zf[1] - zf[0])
    s = 0.0
    volf = 0.0
    for _rep in range(4):
        for kk in range(k1, k2 + 1):
            v = f[min(max(kk, 1), nf)]
            za, zb = zf[kk - 1], zf[kk]
            if za <= z1 and zb >= z2:
                s = s + v
                volf = volf + 1.0
                break
            elif za < z1 and zb > z1:
                s = s + v * (zb - z1) * ssdzf
                volf = volf + (zb - z1) * ssdzf
            elif za >= z1 and zb <= z2:
                s = s + v
                volf = volf + 1.0
            elif za < z2 and zb > z2:
                s = s + v * (z2 - za) * ssdzf
                volf = volf + (z2 - za) * ssdzf
            elif za >= z2:
                break
    return s / volf
