"""Benchmark cases of the mPDeC5 time step and their initial states.

The reference selects its problems through parameters.f90 (InitialCondition,
grid, domain, Gravity, BathymetryFlag; parameters.f90:62-127) and fills cell
averages with a 4x4 Gauss rule (finitevolume.f90:314-330).  The cases below are
new InitialCondition/BathymetryFlag entries in the same style, all periodic:

  vortex    50x50 on [0,4]^2, travelling cyclostrophic vortex, b = 0
  lake      512x256 on [0,2]x[0,1], lake at rest over a Gaussian bump + pulse (WB on)
  lake_dry  the same with a 1.05 bump (dry patch)
  dambreak  1024^2 on [-2,2]^2, h = 1 for r < 0.5, dry (MIN_DEPTH) elsewhere
  island    2048^2 on [0,10]^2, Gaussian island (dry top) + incoming hump
  ensemble  256 problems, sides log-uniform in [64,512], mixed families

Inputs are synthetic (no dataset exists for this path); the initial-condition
fill is driver-side work in the reference and runs here on the host with numpy.
"""
import math

import numpy as np

MIN_DEPTH = 1.0e-6
G = 9.81


def quadrature():
    """4-point Gauss nodes on [-1/2,1/2] and weights (mesh.f90:127-129)."""
    s = math.sqrt(6.0 / 5.0)
    a = math.sqrt(3.0 / 7.0 + 2.0 / 7.0 * s)
    b = math.sqrt(3.0 / 7.0 - 2.0 / 7.0 * s)
    qn = np.array([-(0.5 * a), -(0.5 * b), 0.5 * b, 0.5 * a])
    w1 = (18.0 - math.sqrt(30.0)) / 72.0
    w2 = (18.0 + math.sqrt(30.0)) / 72.0
    qw = np.array([w1, w2, w2, w1])
    return qn, qw


def gauss_coords(x0, h, n):
    """Gauss-node coordinates [n][4] of n cells (mesh.f90:64,70,142)."""
    qn, _ = quadrature()
    c = np.arange(n, dtype=np.float64)
    node = x0 + c * h
    bary = node + 0.5 * h
    return bary[:, None] + qn[None, :] * h


def bathymetry(case, x, y):
    """Gaussian bump b = A exp(-(ax (x-cx)^2 + ay (y-cy)^2)) (SWM_BATHY_GAUSS)."""
    if case.get("bathy_flag", 0) != 3:
        return np.zeros(np.broadcast(x, y).shape)
    A, ax, cx, ay, cy = case["bathy_par"]
    dx, dy = x - cx, y - cy
    return A * np.exp(-(ax * (dx * dx) + ay * (dy * dy)))


def point_state(case, ic, par, x, y):
    """Conservative state (h, hu, hv) at points (x, y) for the new IC ids."""
    g = case["g"]
    if ic == 101:  # vortex: par (cx, cy, eps, ub, vb, R)
        cx, cy, eps, ub, vb, R = par
        rx, ry = (x - cx) / R, (y - cy) / R
        e1 = np.exp(1.0 - (rx * rx + ry * ry))
        h = 1.0 - eps * eps / (4.0 * g) * (e1 * e1)
        return h, h * (ub - eps * ry * e1), h * (vb + eps * rx * e1)
    if ic == 102:  # lake at rest + pulse: par (amp, xlo, xhi)
        amp, xlo, xhi = par
        h = np.maximum(1.0 - bathymetry(case, x, y), MIN_DEPTH)
        h = np.where((x > xlo) & (x < xhi), h + amp, h)
        z = np.zeros_like(h)
        return h, z, z
    if ic == 103:  # dam break: par (cx, cy, radius, h_in)
        cx, cy, R, hin = par
        a, c = x - cx, y - cy
        h = np.where(np.sqrt(a * a + c * c) < R, hin, MIN_DEPTH) + 0.0 * x * y
        z = np.zeros_like(h)
        return h, z, z
    if ic == 104:  # wave over island: par (amp, xc, width)
        amp, xc, w = par
        hs = np.maximum(1.0 - bathymetry(case, x, y), MIN_DEPTH)
        s = (x - xc) / w
        eta = amp * np.exp(-(s * s))
        h = hs + eta
        return h, eta * np.sqrt(g * h), np.zeros_like(h)
    if ic == 105:  # still water: par (level,)
        h = np.maximum(par[0] - bathymetry(case, x, y), MIN_DEPTH)
        z = np.zeros_like(h)
        return h, z, z
    raise ValueError(f"unknown initial condition {ic}")


def cell_averages(case, ic=None, par=None):
    """Cell averages [3][ny][nx] by the 4x4 Gauss rule (finitevolume.f90:314-330)."""
    ic = case["ic"] if ic is None else ic
    par = case["par"] if par is None else par
    nx, ny = case["nx"], case["ny"]
    (x0, y0), (x1, y1) = case["x0"], case["x1"]
    dx, dy = abs(x1 - x0) / nx, abs(y1 - y0) / ny
    X = gauss_coords(x0, dx, nx)  # [nx][4]
    Y = gauss_coords(y0, dy, ny)  # [ny][4]
    _, qw = quadrature()
    U = np.zeros((3, ny, nx))
    for a in range(4):
        for b in range(4):
            w = qw[a] * qw[b]
            st = point_state(case, ic, par, X[None, :, a], Y[:, b, None])
            for v in range(3):
                U[v] = U[v] + w * np.broadcast_to(st[v], (ny, nx))
    return U


def ghosted(planes):
    """Planes [3][ny][nx] -> the reference layout U(1:3,-2:nx+3,-2:ny+3) as a C array
    [ny+6][nx+6][3], ghosts filled periodically (equation.f90:556-776)."""
    _, ny, nx = planes.shape
    jj = (np.arange(-3, ny + 3)) % ny
    ii = (np.arange(-3, nx + 3)) % nx
    return np.ascontiguousarray(planes[:, jj][:, :, ii].transpose(1, 2, 0))


def planes_of(U):
    """Inverse of ghosted(): interior planes [3][ny][nx]."""
    return np.ascontiguousarray(U[3:-3, 3:-3, :].transpose(2, 0, 1))


def vortex_centre(seed):
    """Centre (2,2) jittered by U(-0.05, 0.05)^2 from numpy's default_rng(seed)."""
    d = np.random.default_rng(seed).uniform(-0.05, 0.05, 2)
    return 2.0 + d[0], 2.0 + d[1]


def case(name, seed=0, n=None):
    """Parameters of a named case; n overrides the grid side (parity runs)."""
    if name == "vortex":
        cx, cy = vortex_centre(seed)
        c = dict(nx=50, ny=50, x0=(0.0, 0.0), x1=(4.0, 4.0), g=G, cfl=0.4, tend=0.1,
                 bathy_flag=0, bathy_par=(0, 0, 0, 0, 0), ic=101,
                 par=(cx, cy, 0.5, 1.0, 1.0, 0.4), well_balanced=0)
    elif name in ("lake", "lake_dry"):
        A = 0.8 if name == "lake" else 1.05
        c = dict(nx=512, ny=256, x0=(0.0, 0.0), x1=(2.0, 1.0), g=G, cfl=0.4, tend=0.05,
                 bathy_flag=3, bathy_par=(A, 5.0, 0.9, 50.0, 0.5), ic=102,
                 par=(0.01, 0.05, 0.15), wb_ic=105, wb_par=(1.0,), well_balanced=1)
    elif name == "dambreak":
        c = dict(nx=1024, ny=1024, x0=(-2.0, -2.0), x1=(2.0, 2.0), g=G, cfl=0.4, tend=0.4,
                 bathy_flag=0, bathy_par=(0, 0, 0, 0, 0), ic=103, par=(0.0, 0.0, 0.5, 1.0),
                 well_balanced=0)
    elif name == "island":
        c = dict(nx=2048, ny=2048, x0=(0.0, 0.0), x1=(10.0, 10.0), g=G, cfl=0.4, tend=None,
                 bathy_flag=3, bathy_par=(1.2, 2.0, 5.0, 2.0, 5.0), ic=104, par=(0.3, 2.0, 0.3),
                 well_balanced=0)
    else:
        raise ValueError(name)
    if n is not None:
        ratio = c["ny"] / c["nx"]
        c["nx"], c["ny"] = int(n), max(3, int(round(n * ratio)))
    return c


def ensemble(seed=0, n=256, smin=64, smax=512):
    """Seeded ensemble: side round(exp(U(ln smin, ln smax))), family uniform over
    vortex (eps in U[0.2,0.8]), dam break (radius in U[0.3,0.8]) and Gaussian lake
    (amplitude in U[0.3,1.1]); each family keeps its domain."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        side = int(round(math.exp(rng.uniform(math.log(smin), math.log(smax)))))
        fam = int(rng.integers(0, 3))
        if fam == 0:
            eps = rng.uniform(0.2, 0.8)
            c = case("vortex", n=side)
            cx, cy = 2.0 + rng.uniform(-0.05, 0.05), 2.0 + rng.uniform(-0.05, 0.05)
            c["par"] = (cx, cy, eps, 1.0, 1.0, 0.4)
        elif fam == 1:
            c = case("dambreak", n=side)
            c["par"] = (0.0, 0.0, rng.uniform(0.3, 0.8), 1.0)
        else:
            c = case("lake", n=side)
            A = rng.uniform(0.3, 1.1)
            c["bathy_par"] = (A, 5.0, 0.9, 50.0, 0.5)
            c["well_balanced"] = 0
        c["family"] = ("vortex", "dambreak", "lake")[fam]
        out.append(c)
    return out
