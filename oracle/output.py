"""CPU restatement of the reference's solution output (output.f90), for tests only.

WriteSolutionToDisk / WriteDataToDisk_TECPLOT / WriteDataToDisk_OCTAVE /
WriteMeshToDisk / TIMESTAMP (output.f90:29-395).  Every value is written with the
edit descriptor (SP,ES21.14E2); Python's '%+.14E' is the correctly rounded
conversion of the binary value (ties to even), the same digits C's printf gives.
An exponent that needs three digits does not fit E2 and the field is filled with
asterisks, as a Fortran Ew.dEe field that cannot hold its exponent is.

Parity note: the reference's gfortran runtime could not be run here (no Fortran
compiler), so the byte-level format is restated from the edit descriptors, not
pinned against files the reference wrote.
"""
import math

import numpy as np

VAR_NAMES = ("Depth", "VelocityX", "VelocityY", "Bathymetry")  # parameters.f90:149-152


def es21(x):
    """(SP,ES21.14E2) of one double."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(21)
    if math.isinf(x):
        return ("+Infinity" if x > 0 else "-Infinity").rjust(21)
    s = f"{x:+.14E}"
    return s if len(s) == 21 else "*" * 21


def timestamp(name, t):
    """TIMESTAMP (output.f90:375-395): F15.7 with blanks replaced by zeros."""
    return f"{name}_" + f"{t:15.7f}".replace(" ", "0")


def barycentres(nx, ny, x0, x1):
    """MeshBary (mesh.f90:58-70): MeshNodes(ii-1) + 0.5 Mesh_DX, row-major [ny][nx]."""
    dx = abs(abs(x1[0] - x0[0])) / float(nx)
    dy = abs(abs(x1[1] - x0[1])) / float(ny)
    xs = np.array([(x0[0] + float(i) * dx) + 0.5 * dx for i in range(nx)])
    ys = np.array([(x0[1] + float(j) * dy) + 0.5 * dy for j in range(ny)])
    return np.broadcast_to(xs[None, :], (ny, nx)), np.broadcast_to(ys[:, None], (ny, nx))


def _zero_small(v):
    return 0.0 if abs(v) < 1.0e-70 else v


def tecplot_text(t, nx, ny, x0, x1, planes):
    """WriteDataToDisk_TECPLOT (output.f90:236-305) for planes[4][ny][nx]."""
    head = 'VARIABLES="CoordinateX","CoordinateY"' + "".join(f',"{v}"' for v in VAR_NAMES)
    zone = (f'ZONE T="FV2D",STRANDID=1,SOLUTIONTIME={f"{t:15.8f}".lstrip()}, DATAPACKING=POINT, '
            f"ZONETYPE=ORDERED, I={nx}, J={ny}")
    X, Y = barycentres(nx, ny, x0, x1)
    lines = [head, zone]
    for j in range(ny):
        for i in range(nx):
            vals = [X[j, i], Y[j, i]] + [_zero_small(planes[v][j, i]) for v in range(4)]
            lines.append("".join(es21(v) + "  " for v in vals))
    return "\n".join(lines) + "\n"


def octave_text(planes):
    """WriteDataToDisk_OCTAVE (output.f90:310-370): names in 23-wide fields."""
    head = "".join(v.ljust(23) for v in VAR_NAMES)
    ny, nx = planes[0].shape
    lines = [head]
    for j in range(ny):
        for i in range(nx):
            lines.append("".join(es21(_zero_small(planes[v][j, i])) + "  " for v in range(4)))
    return "\n".join(lines) + "\n"


def mesh_text(nx, ny, x0, x1, d):
    """WriteMeshToDisk (output.f90:190-231), d = 0 (x) or 1 (y)."""
    X, Y = barycentres(nx, ny, x0, x1)
    vals = X[0, :] if d == 0 else Y[:, 0]
    return ("CoordinateX" if d == 0 else "CoordinateY") + "\n" + "".join(es21(v) + "\n" for v in vals)


def cons_to_prim(P):
    """ConsToPrim (equation.f90:912-945) of planes [3][ny][nx]: u = hu / (h + 1e-6/h)."""
    h, hu, hv = P
    with np.errstate(divide="ignore", invalid="ignore"):
        ht = h + 1.0e-6 / h
        return np.stack([h, hu / ht, hv / ht])
