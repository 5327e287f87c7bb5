"""GPU parity of the sm_100a time step against the CPU oracle, through the C ABI.

Bars (from the task statement of the path):
  * FP64_EXACT form: bit-identical RHS, dt, Patankar/Jacobi iterates and full
    steps on flat-bottom cases (no libm call on the path);
  * FP64 form: relative L1 <= 1e-12 per variable after the stated steps;
  * split form: relative L1 <= 1e-6 per variable (FP32 WENO weights);
  * h >= 0, mass conserved to roundoff, lake at rest held exactly.
"""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    """Relative L1 error per variable: sum|a-b| / max(sum|b|, tiny)."""
    return [float(np.abs(a[v] - b[v]).sum() / max(np.abs(b[v]).sum(), 1e-300))
            for v in range(a.shape[0])]


def make_pair(swm, name, n=None, seed=0, precision="fp64", solver="csr", block=0,
              timescheme=5, compat=0, maxiter=1000, use_graph=1, wb_pulse=True):
    c = cases.case(name, seed=seed, n=n)
    op = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                       timescheme=timescheme, bathy_flag=c["bathy_flag"],
                       bathy_par=c["bathy_par"], well_balanced=c["well_balanced"],
                       jacobi_maxiter=maxiter, mpdec2_compat=compat)
    o = O.Oracle(op)
    planes = cases.cell_averages(c) if wb_pulse else cases.cell_averages(c, c["wb_ic"], c["wb_par"])
    s = swm.Solver(nx=c["nx"], ny=c["ny"], x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                   timescheme=timescheme, bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                   well_balanced=c["well_balanced"], precision=precision, solver=solver,
                   jacobi_block=block, mpdec2_compat=compat, jacobi_maxiter=maxiter,
                   use_graph=use_graph)
    if c["well_balanced"]:
        wb = cases.cell_averages(c, c["wb_ic"], c["wb_par"])
        o.init_wb_planes(wb)
        s.set_wb_state(cases.ghosted(wb))
    o.set_planes(planes)
    s.set_planes(planes)
    return c, o, s


@pytest.mark.parametrize("name,n", [("vortex", 48), ("dambreak", 40)])
def test_rhs_exact_bitwise(gpu, name, n):
    c, o, s = make_pair(gpu, name, n)
    U = o.get_state()[0]
    ref = o.rhs()
    got = s.debug_rhs(U)
    for key in ("FX", "FY"):
        assert np.array_equal(got[key], ref[key]), key
    assert np.array_equal(got["Ut"], ref["Ut"])  # Ut(1) too (explicit schemes)
    assert np.array_equal(got["S"], ref["S"])


@pytest.mark.parametrize("name", ["lake", "island"])
def test_rhs_exact_bathymetry(gpu, name):
    # the analytic bathymetry gradient is tabulated with the host libm, so the FP64
    # form's source term is bit-identical too (WB subtraction included for the lake)
    c, o, s = make_pair(gpu, name, 64)
    ref = o.rhs()
    got = s.debug_rhs(o.get_state()[0])
    for key in ("FX", "FY", "S"):
        assert np.array_equal(got[key], ref[key]), key
    assert np.array_equal(got["Ut"], ref["Ut"])  # Ut(1) too (explicit schemes)


# fp64_fma: where a stencil varies by < ~1e-7 the reference's smoothness indicators
# are rounding noise, so contracted arithmetic may move face values by that much.
@pytest.mark.parametrize("precision,tol", [("fp64_fma", 5e-7), ("split", 2e-6)])
@pytest.mark.parametrize("name,n", [("vortex", 48), ("island", 64)])
def test_rhs_forms_close(gpu, precision, tol, name, n):
    c, o, s = make_pair(gpu, name, n, precision=precision)
    ref = o.rhs()
    got = s.debug_rhs(o.get_state()[0])
    for key in ("FX", "FY"):
        err = np.abs(got[key] - ref[key]).max()
        assert err <= tol * max(np.abs(ref[key]).max(), 1.0), (key, err)
    # Ut is a flux difference over dx: its error scale is (flux error) / dx
    dx = (c["x1"][0] - c["x0"][0]) / c["nx"]
    f_scale = max(np.abs(ref["FX"]).max(), np.abs(ref["FY"]).max(), 1.0)
    assert np.abs(got["Ut"] - ref["Ut"]).max() <= 4 * tol * f_scale / dx


# The reference's other bathymetries (equation.f90:430-438) with their reference
# initial states: the sin/cos bottom (separable: the split and FMA forms take the
# per-column/row factors) and the bump (the full gradient table in every form).
@pytest.mark.parametrize("bathy,ic,dom", [(1, 2, ((0.0, 0.0), (1.0, 1.0))),
                                          (2, 6, ((-3.0, -1.5), (3.0, 2.5)))])
@pytest.mark.parametrize("precision,tol", [("fp64", 0.0), ("fp64_fma", 5e-7), ("split", 2e-6)])
def test_rhs_other_bathymetries(gpu, bathy, ic, dom, precision, tol):
    nx, ny = 40, 36
    o = O.Oracle(O.make_params(nx, ny, dom[0], dom[1], g=9.81, cfl=0.4, bathy_flag=bathy))
    o.fill_ic(ic)
    s = gpu.Solver(nx=nx, ny=ny, x0=dom[0], x1=dom[1], g=9.81, cfl=0.4, bathy_flag=bathy,
                   bathy_par=(0.0,) * 5, precision=precision, solver="stencil", jacobi_block=4)
    ref = o.rhs()
    got = s.debug_rhs(o.get_state()[0])
    if tol == 0.0:
        for key in ("FX", "FY", "S", "Ut"):
            assert np.array_equal(got[key], ref[key]), key
        return
    f_scale = max(np.abs(ref["FX"]).max(), np.abs(ref["FY"]).max(), 1.0)
    for key in ("FX", "FY"):
        assert np.abs(got[key] - ref[key]).max() <= tol * f_scale, key
    s_scale = max(np.abs(ref["S"]).max(), 1.0)
    assert np.abs(got["S"] - ref["S"]).max() <= tol * s_scale
    dx = (dom[1][0] - dom[0][0]) / nx
    assert np.abs(got["Ut"] - ref["Ut"]).max() <= 4 * tol * f_scale / dx


def test_timestep_bitwise(gpu):
    c, o, s = make_pair(gpu, "vortex", 50)
    assert s.timestep() == o.timestep()


def random_patankar_system(n_cells, seed):
    """A Patankar-like M-matrix in the reference CSR layout: off-diagonals <= 0,
    diagonal 1 + (column production), right-hand side > 0."""
    rng = np.random.default_rng(seed)
    mass = -0.1 * rng.random((n_cells, 5))
    mass[:, 2] = 0.0
    diag = 1.0 + 0.4 * rng.random(n_cells)
    rhs = 0.5 + rng.random(n_cells)
    return mass.reshape(-1).copy(), diag, rhs


@pytest.mark.parametrize("solver,block", [("csr", 0), ("stencil", 1), ("stencil", 2),
                                          ("stencil", 4), ("stencil", 8)])
def test_jacobi_bitwise(gpu, solver, block):
    c, o, s = make_pair(gpu, "vortex", 70, solver=solver, block=block)
    mass, diag, rhs = random_patankar_system(70 * 70, 3)
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k == k_ref
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("n", [96, 100])
@pytest.mark.parametrize("block", [1, 2, 4])
def test_jacobi_bitwise_wide(gpu, n, block):
    # grids wider than one haloed tile, with 16-byte pair loads (even nx); 100 is not a
    # multiple of the 64-wide tiles, so edge tiles hang over the grid
    c, o, s = make_pair(gpu, "vortex", n, solver="stencil", block=block)
    mass, diag, rhs = random_patankar_system(n * n, 11)
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k == k_ref
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("name", ["vortex", "dambreak"])
def test_steps_exact_bitwise_wide(gpu, name):
    c, o, s = make_pair(gpu, name, 96, solver="stencil", block=4)
    for _ in range(2):
        dt = o.timestep()
        assert s.timestep() == dt
        o.step(0.0, dt)
        s.step(0.0, dt)
    assert np.array_equal(s.get_planes(), o.get_planes())
    assert list(s.stats()["jacobi_iters"][:13]) == list(o.last_jacobi_iters()[:13])


@pytest.mark.parametrize("nx,ny", [(65, 17), (66, 33), (129, 18), (130, 47), (67, 31)])
@pytest.mark.parametrize("block", [2, 4, 8])
def test_jacobi_bitwise_ragged_tiles(gpu, nx, ny, block):
    # edge tiles 1, 2, 3 columns wide and 1, 2, 15 rows high (64x16 tiles) hanging
    # over the grid's edge, even and odd row pitches; a slowly converging system, so
    # that every pass runs its full block of sweeps
    c = cases.case("vortex", n=nx)
    o = O.Oracle(O.make_params(nx, ny, c["x0"], c["x1"], g=c["g"], cfl=c["cfl"]))
    s = gpu.Solver(nx=nx, ny=ny, x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                   precision="fp64", solver="stencil", jacobi_block=block)
    rng = np.random.default_rng(nx * 1000 + ny)
    mass = -0.24 * rng.random((nx * ny, 5))
    mass[:, 2] = 0.0
    diag = 1.0 + 0.05 * rng.random(nx * ny)
    rhs = 0.5 + rng.random(nx * ny)
    mass = mass.reshape(-1).copy()
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k_ref > 3 * block
    assert k == k_ref
    assert np.array_equal(got, ref)
    s.close()


@pytest.mark.parametrize("maxiter", [1, 2, 3, 5, 6, 7, 9, 1000])
@pytest.mark.parametrize("block", [2, 4])
def test_jacobi_planned_passes_vs_maxiter(gpu, maxiter, block):
    # passes are sized from the residual decay and may write the destination
    # directly; whatever the plan, the iterate, the stop index and the maxIter
    # warning must be those of the reference's one-sweep-at-a-time loop
    c, o, s = make_pair(gpu, "vortex", 96, maxiter=maxiter, solver="stencil", block=block)
    mass, diag, rhs = random_patankar_system(96 * 96, 17)
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k == k_ref
    assert rc == (1 if k_ref == maxiter else 0)
    assert np.array_equal(got, ref)


def test_jacobi_maxiter_warning(gpu):
    c, o, s = make_pair(gpu, "vortex", 40, maxiter=3, solver="stencil", block=2)
    mass, diag, rhs = random_patankar_system(40 * 40, 5)
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k == k_ref == 3 and rc == 1
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("solver,block", [("csr", 0), ("stencil", 4)])
def test_step_exact_bitwise(gpu, solver, block):
    c, o, s = make_pair(gpu, "vortex", 50, solver=solver, block=block)
    dt = o.timestep()
    assert s.timestep() == dt
    o.step(0.0, dt)
    assert s.step(0.0, dt) == 0
    assert np.array_equal(s.get_planes(), o.get_planes())
    assert s.stats()["jacobi_iters"] == o.last_jacobi_iters()


def test_step_exact_bitwise_dambreak(gpu):
    c, o, s = make_pair(gpu, "dambreak", 48)
    for step in range(3):
        dt = o.timestep()
        assert s.timestep() == dt
        o.step(0.0, dt)
        s.step(0.0, dt)
    assert np.array_equal(s.get_planes(), o.get_planes())


@pytest.mark.parametrize("precision,solver,block,tol", [
    ("fp64", "csr", 0, 0.0),
    ("fp64", "stencil", 4, 0.0),
    ("fp64_fma", "stencil", 4, 1e-7),
    ("split", "stencil", 4, 1e-6),
])
def test_vortex_to_tend(gpu, precision, solver, block, tol):
    c, o, s = make_pair(gpu, "vortex", None, seed=1, precision=precision, solver=solver,
                        block=block)
    n_o, t_o = o.run(c["tend"], 4)
    n_s, t_s = s.run(c["tend"], 4)
    assert n_o == n_s and abs(t_o - 0.1) < 1e-10
    err = rel_l1(s.get_planes(), o.get_planes())
    assert max(err) <= tol, err


def test_lake_at_rest_exact(gpu):
    # lake at rest over the Gaussian bump, WB on: U(t) == U(0) exactly
    for precision in ("fp64", "split", "fp64_fma"):
        c, o, s = make_pair(gpu, "lake", 64, precision=precision, solver="stencil", block=4,
                            wb_pulse=False)
        U0 = s.get_planes().copy()
        for _ in range(3):
            s.step(0.0, s.timestep())
        assert np.array_equal(s.get_planes(), U0), precision


def test_lake_pulse_parity(gpu):
    c, o, s = make_pair(gpu, "lake", 64, precision="fp64", solver="stencil", block=4)
    for _ in range(4):
        dt = o.timestep()
        o.step(0.0, dt)
        s.step(0.0, dt)
    assert np.array_equal(s.get_planes(), o.get_planes())


def test_dambreak_positivity_mass(gpu):
    c, o, s = make_pair(gpu, "dambreak", 96, precision="split", solver="stencil", block=4)
    m0, _ = s.summary()
    for _ in range(10):
        s.step(0.0, s.timestep())
    m1, hmin = s.summary()
    assert hmin > 0.0
    assert abs(m1 - m0) <= 1e-12 * m0


def test_mpdec2(gpu):
    c, o, s = make_pair(gpu, "vortex", 40, timescheme=7)
    for _ in range(2):
        dt = o.timestep()
        assert s.timestep() == dt
        o.step(0.0, dt)
        s.step(0.0, dt)
    assert np.array_equal(s.get_planes(), o.get_planes())


def test_mpdec2_compat_reproduces_reference_read(gpu):
    # mPDeC2 passes Up(:,1,:,:) (extent 4) to hp(2,nx,ny) (timediscretization.f90:634,784):
    # half of the depths read are the never-written Up(3:4) zeros; both sides reproduce it,
    # including the resulting non-finite cells
    c, o, s = make_pair(gpu, "vortex", 40, timescheme=7, compat=1)
    dt = o.timestep()
    o.step(0.0, dt)
    ref = o.get_planes()
    try:
        rc = s.step(0.0, dt)
    except gpu.SwmError as e:  # the step reports the non-finite cells it produced
        rc = e.code
    assert rc == (0 if np.all(np.isfinite(ref)) else -3)
    assert np.array_equal(s.get_planes(), ref, equal_nan=True)


def test_graph_and_eager_identical(gpu):
    outs = []
    for g in (0, 1):
        c, o, s = make_pair(gpu, "island", 64, precision="split", solver="stencil", block=4,
                            use_graph=g)
        for _ in range(2):
            s.step(0.0, s.timestep())
        outs.append(s.get_planes())
    assert np.array_equal(outs[0], outs[1])


def test_csr_and_stencil_steps_identical(gpu):
    outs = []
    for solver, block in (("csr", 0), ("stencil", 1), ("stencil", 4), ("stencil", 8)):
        c, o, s = make_pair(gpu, "island", 80, precision="fp64", solver=solver, block=block)
        for _ in range(2):
            s.step(0.0, s.timestep())
        outs.append((s.get_planes(), s.stats()["jacobi_iters"]))
    for P, it in outs[1:]:
        assert np.array_equal(P, outs[0][0])
        assert it == outs[0][1]


def test_state_roundtrip_and_v(gpu):
    c, o, s = make_pair(gpu, "vortex", 20)
    U = o.get_state()[0]
    s.set_state(cases.ghosted(cases.planes_of(U)))
    U2, V2 = s.get_state(with_v=True)
    assert np.array_equal(cases.planes_of(U2), cases.planes_of(U))
    h = U2[..., 0]
    assert np.allclose(V2[..., 1], U2[..., 1] / (h + 1e-6 / h), rtol=0, atol=1e-15)


def test_nan_state_rejected(gpu):
    c, o, s = make_pair(gpu, "vortex", 16)
    P = s.get_planes()
    P[0, 3, 3] = np.nan
    s.set_planes(P)
    with pytest.raises(gpu.SwmError) as e:
        s.timestep()
    assert e.value.code == -3


@pytest.mark.parametrize("precision", ["fp64", "split", "fp64_fma"])
@pytest.mark.parametrize("name,n", [("vortex", 64), ("island", 96), ("lake", 80)])
def test_rhs_tma_and_wrapped_loads_identical(gpu, precision, name, n):
    # tiles whose haloed box lies inside the grid are staged by TMA, the seam tiles by
    # wrapped loads; loading every tile the wrapped way must give the same bits
    c, o, s = make_pair(gpu, name, n, precision=precision, solver="stencil", block=4)
    U = o.get_state()[0]
    s.set_tma(True)
    a = s.debug_rhs(U)
    s.set_tma(False)
    b = s.debug_rhs(U)
    for key in ("Ut", "FX", "FY", "S"):
        assert np.array_equal(a[key], b[key]), key
    if precision == "fp64":
        ref = o.rhs()
        for key in ("Ut", "FX", "FY", "S"):
            assert np.array_equal(a[key], ref[key]), key


def test_steps_with_and_without_tma_identical(gpu):
    outs = []
    for tma in (True, False):
        c, o, s = make_pair(gpu, "island", 128, precision="split", solver="stencil", block=4)
        s.set_tma(tma)
        for _ in range(3):
            s.step(0.0, s.timestep())
        outs.append(s.get_planes())
    assert np.array_equal(outs[0], outs[1])
