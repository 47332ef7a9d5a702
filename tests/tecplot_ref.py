"""Test infrastructure: TecPlot_CellCenter (TecPlot_ASCII.f90:2-86) restated
in Python from a simulation state (the oracle's, through the same accessors
as the library's: leaves, topology, download_block, physics), with the
Fortran edit descriptors it uses (F10.3, E14.6, I6, I7, format reversion),
to check the library's writer byte for byte. Not used by the library.

The two list-directed lines of the reference are processor-dependent; they
are restated as the library documents them: one leading blank, the time as
%.17g."""
import math

import numpy as np


def fortran_i(v, w):
    """Iw: right-justified, asterisks when it does not fit."""
    s = f"{int(v):{w}d}"
    return "*" * w if len(s) > w else s


def fortran_f(v, w=10, d=3):
    """Fw.d (correctly rounded decimal of the binary value)."""
    s = f"{v:{w}.{d}f}"
    return "*" * w if len(s) > w else s


def fortran_e(v, w=14, d=6):
    """Ew.d, scale factor 0: [-]0.d1..dd followed by E+ee, or by +eee
    without the E when the exponent needs three digits."""
    if math.isnan(v):
        body = "NaN"
    elif math.isinf(v):
        body = "-Infinity" if v < 0 else "Infinity"
    else:
        a = abs(v)
        if a == 0.0:
            digs, e10 = "0" * d, 0
        else:
            mant, ex = f"{a:.{d - 1}e}".split("e")
            digs, e10 = mant.replace(".", ""), int(ex) + 1
        sign = "-" if math.copysign(1.0, v) < 0 else ""
        ae = abs(e10)
        es = "-" if e10 < 0 else "+"
        expo = f"E{es}{ae:02d}" if ae <= 99 else f"{es}{ae:03d}"
        body = f"{sign}0.{digs}{expo}"
    return "*" * w if len(body) > w else body.rjust(w)


def records(items, per):
    """Format reversion: `per` items a record, the last one shorter."""
    return "".join("".join(items[i:i + per]) + "\n" for i in range(0, len(items), per))


def tecplot_text(sim, params, t):
    nx, ny = params.nx, params.ny
    L0 = params.dx0 * nx
    D = 2.0 * params.radius
    ph = sim.physics()
    topo = sim.topology()
    leaves = [int(b) for b in sim.leaves()]
    X, Y, cn, u, v, p = [], [], [], [], [], []
    for b in leaves:
        f = sim.download_block(b)
        dx, bi, bj = (int(topo[k][b - 1]) for k in ("dx", "bi", "bj"))
        for J in range(1, ny + 2):
            for I in range(1, nx + 2):
                X.append(bi * dx * nx + dx * (I - 1))
                Y.append(bj * dx * ny + dx * (J - 1))
        C = np.asarray(f["C"]).reshape((nx + 4, ny + 4), order="F")  # C(-1:nx+2, -1:ny+2)
        s = ((C[1:nx + 2, 1:ny + 2] + C[2:nx + 3, 1:ny + 2]) + C[1:nx + 2, 2:ny + 3]) \
            + C[2:nx + 3, 2:ny + 3]
        cn.extend((0.25 * s - 0.5).ravel(order="F").tolist())
        u.extend(np.asarray(f["Ux"]).ravel(order="F").tolist())
        v.extend(np.asarray(f["Uy"]).ravel(order="F").tolist())
        P = np.asarray(f["P"]).ravel(order="F")
        p.extend((((P * 0.5) * D) / ph.sigma).tolist())
    Nn, Ne = len(X), len(u)
    out = [" Variables = X, Y, Ux, Uy, C, P\n",
           "Zone N =" + fortran_i(Nn, 6) + ", E =" + fortran_i(Ne, 6)
           + ", ZONETYPE=FEquadrilateral, DATAPACKING=Block\n",
           f' VARLOCATION=([3,4,6]=CELLCENTERED), T = "{t * math.sqrt(ph.gy / D):.17g}"\n']
    l0 = np.float32(L0)
    out.append(records([fortran_f(float(np.float32(x) / l0)) for x in X], 9))
    out.append(records([fortran_f(float(np.float32(y) / l0)) for y in Y], 9))
    out.append(records([fortran_e(a) for a in u], 8))
    out.append(records([fortran_e(a) for a in v], 8))
    out.append(records([fortran_e(a) for a in cn], 9))
    out.append(records([fortran_e(a) for a in p], 8))
    conn = []
    for m in range(len(leaves)):
        for J in range(ny):
            for I in range(nx):
                N = m * (nx + 1) * (ny + 1) + J * (nx + 1) + I + 1
                conn += [N, N + 1, N + 1 + nx + 1, N + nx + 1]
    out.append(records([fortran_i(k, 7) for k in conn], 8))
    return "".join(out)
