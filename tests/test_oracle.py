"""Known answers of the CPU oracle, derived from the reference source.

The reference ships no golden vectors and no Fortran compiler exists here, so
the restatement is pinned by properties the Fortran code has by construction:
quadrature and DeC tables (mesh.f90:127-129, timediscretization.f90:491-511),
polynomial exactness of the WENO5 stencils (reconstruction.f90:673-1136),
well-balancing of the lake at rest (finitevolume.f90:485-489), conservation and
positivity of the Patankar update (timediscretization.f90:771-924), the CSR
layout (finitevolume.f90:219-271), the Jacobi stopping rule
(jacobi_iteration.f90:52-87), and high-order convergence on a vortex whose exact
solution is a translation.
"""
import math

import numpy as np
import pytest

import cases
import oracle as O


def test_quadrature_tables():
    qn, qw = O.quadrature()
    assert abs(qw.sum() - 1.0) < 1e-15
    assert np.allclose(qn, -qn[::-1], rtol=0, atol=0)
    # exact for polynomials up to degree 7 on [-1/2, 1/2]
    for k in range(8):
        exact = 0.0 if k % 2 else (0.5 ** k) / (k + 1)
        assert abs((qw * qn ** k).sum() - exact) < 1e-15


def test_theta_rows_sum_to_beta():
    th, beta = O.theta_mpdec5()
    assert np.allclose(th.sum(axis=1), beta, rtol=0, atol=2e-16)
    assert np.allclose(th[3], [1 / 12, 5 / 12, 5 / 12, 1 / 12], rtol=0, atol=1e-16)
    assert np.all(th[0] == 0.0)


def test_weno_first_sweep_exact_for_quadratics():
    # cell averages of f = a + b x + c x^2 on unit cells centred at k: a + b k + c (k^2 + 1/12)
    rng = np.random.default_rng(0)
    for _ in range(50):
        a, b, c = rng.normal(size=3)
        k = np.arange(-2, 3)
        q = a + b * k + c * (k * k + 1.0 / 12.0)
        wm, wp = O.weno5_first(q)
        f = lambda x: a + b * x + c * x * x
        assert abs(wm - f(-0.5)) < 1e-13 and abs(wp - f(0.5)) < 1e-13


def test_weno_second_sweep_exact_for_quadratics():
    qn, _ = O.quadrature()
    rng = np.random.default_rng(1)
    for _ in range(50):
        a, b, c = rng.normal(size=3)
        k = np.arange(-2, 3)
        q = a + b * k + c * (k * k + 1.0 / 12.0)
        w = O.weno5_second(q)
        assert np.allclose(w, a + b * qn + c * qn * qn, rtol=0, atol=1e-13)


def test_weno_constant_preserved():
    for v in (1e-6, 0.7, 1.0, 3.3):
        wm, wp = O.weno5_first(np.full(5, v))
        assert abs(wm - v) <= 4e-16 * v and abs(wp - v) <= 4e-16 * v
        assert np.allclose(O.weno5_second(np.full(5, v)), v, rtol=4e-16, atol=0)


def test_patankar_div():
    assert O.patankar_div(3.0, 0.5e-6) == 0.0
    assert O.patankar_div(3.0, 2.0) == 2.0 * 2.0 * 3.0 / (4.0 + 4.0)
    h = 1e-3  # h^2 < MIN_DEPTH: denominator h^2 + 1e-6
    assert O.patankar_div(1.0, h) == 2.0 * h * 1.0 / (h * h + 1e-6)


def make(name, n=None, **kw):
    c = cases.case(name, n=n)
    c.update(kw)
    p = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                      well_balanced=c["well_balanced"],
                      timescheme=c.get("timescheme", 5))
    o = O.Oracle(p)
    if c["well_balanced"]:
        o.init_wb_planes(cases.cell_averages(c, c["wb_ic"], c["wb_par"]))
    return c, o


def test_csr_pattern_is_reference_layout():
    c, o = make("vortex", 7)
    rs, cols = o.csr_pattern()
    nx = ny = 7
    N = nx * ny
    assert np.array_equal(rs, 5 * np.arange(1, N + 2) - 4)
    ge = lambda i, j: ((j - 1) % ny) * nx + ((i - 1) % nx) + 1
    exp = []
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            exp += [ge(i, j - 1), ge(i - 1, j), ge(i, j), ge(i + 1, j), ge(i, j + 1)]
    assert np.array_equal(cols, exp)


def test_jacobi_stopping_rule():
    c, o = make("vortex", 8)
    N = 64
    mass = np.zeros(5 * N)
    diag = np.full(N, 2.0)
    rhs = np.linspace(1.0, 2.0, N)
    sol, k = o.jacobi(mass, diag, rhs)
    # x1 = b/2 (change mean|b/2 - b| > tol), x2 = x1 (change 0 <= tol): stops at k = 2
    assert k == 2 and np.array_equal(sol, rhs / 2.0)


def test_jacobi_maxiter():
    p = O.make_params(8, 8, (0, 0), (1, 1), jacobi_maxiter=7, jacobi_tol=0.0)
    o = O.Oracle(p)
    rng = np.random.default_rng(2)
    mass = -0.1 * rng.random(5 * 64)
    mass[2::5] = 0.0
    sol, k = o.jacobi(mass, 1.0 + rng.random(64), 1.0 + rng.random(64))
    assert k == 7


def test_lake_at_rest_reference_ic2_well_balanced():
    # reference IC 2 with BathymetryFlag 1 and -DWELLBALANCED (parameters.f90:73-81)
    p = O.make_params(16, 16, (0, 0), (1, 1), g=9.81, cfl=1.0, bathy_flag=1, well_balanced=1)
    o = O.Oracle(p)
    o.init_wb(2)
    o.fill_ic(2)
    U0 = o.get_planes()
    for _ in range(2):
        o.step(0.0, o.timestep())
    assert np.array_equal(o.get_planes(), U0)


def test_lake_without_wb_is_not_at_rest():
    p = O.make_params(16, 16, (0, 0), (1, 1), g=9.81, cfl=1.0, bathy_flag=1, well_balanced=0)
    o = O.Oracle(p)
    o.fill_ic(2)
    U0 = o.get_planes()
    o.step(0.0, o.timestep())
    assert np.abs(o.get_planes()[1] - U0[1]).max() > 1e-8


def test_dambreak_mass_and_positivity():
    c, o = make("dambreak", 32)
    o.set_planes(cases.cell_averages(c))
    m0 = o.get_planes()[0].sum()
    for _ in range(6):
        o.step(0.0, o.timestep())
    P = o.get_planes()
    assert P[0].min() > 0.0
    assert abs(P[0].sum() - m0) <= 1e-13 * m0


def test_vortex_convergence_order():
    # the vortex is an exact travelling solution: error vs the translated IC
    T = 0.05
    errs = []
    for n in (20, 40):
        c = cases.case("vortex", n=n)
        c["par"] = (2.0, 2.0, 0.5, 1.0, 1.0, 0.4)
        p = O.make_params(n, n, c["x0"], c["x1"], g=c["g"], cfl=c["cfl"])
        o = O.Oracle(p)
        o.set_planes(cases.cell_averages(c))
        o.run(T, 1)
        ex = cases.cell_averages(c, par=(2.0 + T, 2.0 + T, 0.5, 1.0, 1.0, 0.4))
        errs.append(np.abs(o.get_planes()[0] - ex[0]).sum() * (4.0 / n) ** 2)
    assert math.log2(errs[0] / errs[1]) > 2.5


@pytest.mark.slow
def test_vortex_convergence_order_fine():
    T = 0.05
    errs = []
    for n in (40, 80):
        c = cases.case("vortex", n=n)
        c["par"] = (2.0, 2.0, 0.5, 1.0, 1.0, 0.4)
        p = O.make_params(n, n, c["x0"], c["x1"], g=c["g"], cfl=c["cfl"])
        o = O.Oracle(p)
        o.set_planes(cases.cell_averages(c))
        o.run(T, 1)
        ex = cases.cell_averages(c, par=(2.0 + T, 2.0 + T, 0.5, 1.0, 1.0, 0.4))
        errs.append(np.abs(o.get_planes()[0] - ex[0]).sum() * (4.0 / n) ** 2)
    assert math.log2(errs[0] / errs[1]) > 4.0


def test_driver_loop_hits_output_times():
    c, o = make("vortex", 12)
    o.set_planes(cases.cell_averages(c))
    steps, t = o.run(0.1, 4)
    assert abs(t - 0.1) < 1e-10 and steps >= 4


def test_mpdec2_runs_and_compat_differs():
    outs = []
    for compat in (0, 1):
        p = O.make_params(12, 12, (0, 0), (4, 4), timescheme=7, mpdec2_compat=compat)
        o = O.Oracle(p)
        c = cases.case("vortex", n=12)
        o.set_planes(cases.cell_averages(c))
        o.step(0.0, o.timestep())
        outs.append(o.get_planes())
    assert np.all(np.isfinite(outs[0]))
    assert not np.array_equal(outs[0], outs[1], equal_nan=True)


def test_l1_error_postprocessing():
    # PostProcessing (postprocessing.f90:23-60): zero on the exact cell averages, and a
    # perturbation delta of one cell shows up as delta * dx * dy
    c = cases.case("vortex", n=24)
    o = O.Oracle(O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"]))
    o.fill_ic(c["ic"], c["par"])
    assert np.array_equal(o.l1_error(c["ic"], c["par"]), np.zeros(3))
    P = o.get_planes()
    P[1, 3, 5] += 0.25
    o.set_planes(P)
    dx = (c["x1"][0] - c["x0"][0]) / c["nx"]
    dy = (c["x1"][1] - c["x0"][1]) / c["ny"]
    l1 = o.l1_error(c["ic"], c["par"])
    assert l1[0] == 0.0 and l1[2] == 0.0
    assert abs(l1[1] - 0.25 * dx * dy) <= 1e-15
    # the reference vortex (case 1) moves with (2, 3): at t = sx/2 it is displaced
    r = O.Oracle(O.make_params(32, 32, (0.0, 0.0), (4.0, 4.0)))
    r.fill_ic(1)
    assert np.all(r.l1_error(1, t=0.0) == 0.0)
    assert r.l1_error(1, t=0.5)[0] > 1e-3
    assert np.allclose(r.l1_error(1, t=4.0 / 2.0 * 2), 0.0, atol=1e-12)  # period 4 in x and y


def test_explicit_schemes_oracle():
    # forward Euler is U + dt Ut with Ut(1) from the mass fluxes (build without
    # PATANKAR); every explicit scheme conserves mass exactly on a periodic grid and
    # the high-order ones agree with each other far better than with Euler
    c = cases.case("vortex", n=24)
    P0 = cases.cell_averages(c)
    res = {}
    for ts in (1, 2, 3, 4):
        o = O.Oracle(O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                                   timescheme=ts))
        o.set_planes(P0)
        if ts == 1:
            Ut = o.rhs()["Ut"]                     # (ny, nx, 3) interior RHS
            o.set_planes(P0)
        dt = 0.25 * o.timestep()
        o.step(0.0, dt)
        P = o.get_planes()
        if ts == 1:
            assert np.array_equal(P, P0 + np.moveaxis(Ut, -1, 0) * dt)
        assert abs(P[0].sum() - P0[0].sum()) <= 1e-12 * P0[0].sum()
        res[ts] = P
    d_hi = max(np.abs(res[a] - res[b]).max() for a, b in ((2, 3), (3, 4), (2, 4)))
    d_lo = np.abs(res[1] - res[3]).max()
    assert d_hi < 1e-2 * d_lo, (d_hi, d_lo)


def test_mpeuler_is_one_mpdec2_correction():
    # mPEuler (KCorr 1) and mPDeC2 (KCorr 2): both keep h >= 0 on a dry dam break and
    # differ by mPDeC2's second correction
    c = cases.case("dambreak", n=24)
    P0 = cases.cell_averages(c)
    out = {}
    for ts in (6, 7):
        o = O.Oracle(O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                                   timescheme=ts))
        o.set_planes(P0)
        o.step(0.0, o.timestep())
        out[ts] = o.get_planes()
        assert out[ts][0].min() >= 0.0
    assert not np.array_equal(out[6], out[7])
    assert abs(out[6][0].sum() - out[7][0].sum()) <= 1e-12 * out[7][0].sum()  # mass


def test_output_formatting_restatement():
    # (SP,ES21.14E2) of output.f90: sign always, 15 correctly rounded digits (ties to
    # even on the exact binary value), two exponent digits or a field of asterisks
    import output as OUT
    assert OUT.es21(1.0) == "+1.00000000000000E+00"
    assert OUT.es21(-0.0) == "-0.00000000000000E+00"
    assert OUT.es21(123.456) == "+1.23456000000000E+02"
    assert OUT.es21(1.0 + 2.0**-15) == "+1.00003051757812E+00"       # exact tie: even
    assert OUT.es21(1.0 + 3 * 2.0**-15) == "+1.00009155273438E+00"   # exact tie: up
    assert OUT.es21(9.9999999999999995) == "+1.00000000000000E+01"
    assert OUT.es21(1e-100) == "*" * 21 and OUT.es21(1e100) == "*" * 21
    assert OUT.es21(float("nan")).strip() == "NaN"
    assert OUT.timestamp("SOLUTION_TEC", 0.1) == "SOLUTION_TEC_0000000.1000000"
    txt = OUT.tecplot_text(0.25, 2, 1, (0.0, 0.0), (2.0, 1.0),
                           [np.ones((1, 2)), np.zeros((1, 2)), np.full((1, 2), 1e-80),
                            np.full((1, 2), -0.5)])
    lines = txt.splitlines()
    assert lines[0] == 'VARIABLES="CoordinateX","CoordinateY","Depth","VelocityX","VelocityY","Bathymetry"'
    assert lines[1] == ('ZONE T="FV2D",STRANDID=1,SOLUTIONTIME=0.25000000, DATAPACKING=POINT, '
                        'ZONETYPE=ORDERED, I=2, J=1')
    assert lines[2].split() == ["+5.00000000000000E-01", "+5.00000000000000E-01",
                                "+1.00000000000000E+00", "+0.00000000000000E+00",
                                "+0.00000000000000E+00", "-5.00000000000000E-01"]
    assert len(lines[2]) == 6 * 23
