"""Initial conditions, well-balanced initialisation and the L1 error on the device
(swm_fill_ic / swm_init_wb_ic / swm_l1_error) against the oracle's restatement of
FillInitialConditions (finitevolume.f90:281-333), InitializeWBVariables (:339-396)
and PostProcessing (postprocessing.f90:23-60).

The device evaluates ExactFunction with CUDA's transcendental functions and the
oracle with the host libm, so cell averages agree to the last few bits (tolerance
below); everything downstream of a shared state is compared bit for bit elsewhere."""
import numpy as np
import pytest

import cases
import oracle as O


pytestmark = pytest.mark.gpu

# |device - host| <= RTOL * max(|host|, 1): a few ulps of the O(1) states
RTOL = 1e-13


def _solver(swm, c, precision="fp64"):
    return swm.Solver(nx=c["nx"], ny=c["ny"], x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                      well_balanced=c["well_balanced"], precision=precision, solver="stencil",
                      jacobi_block=4)


def _oracle(c):
    return O.Oracle(O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                                  bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                                  well_balanced=c["well_balanced"]))


def _close(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))


@pytest.mark.parametrize("name,n", [("vortex", 50), ("lake", 64), ("dambreak", 48),
                                    ("island", 96)])
def test_fill_benchmark_cases(gpu, name, n):
    c = cases.case(name, n=n)
    s, o = _solver(gpu, c), _oracle(c)
    s.fill_ic(c["ic"], c["par"])
    o.fill_ic(c["ic"], c["par"])
    err = _close(s.get_planes(), o.get_planes())
    assert err <= RTOL, err


@pytest.mark.parametrize("ic,bathy,dom", [
    (1, 0, ((0.0, 0.0), (4.0, 4.0))),      # smooth vortex (equation.f90:109-133)
    (2, 0, ((0.0, 0.0), (1.0, 1.0))),      # sin/cos lake
    (3, 2, ((-3.0, -1.5), (3.0, 2.5))),    # perturbed lake over the bump
    (4, 0, ((0.0, 0.0), (20.0, 20.0))),    # dam break (r <= 7)
    (5, 0, ((0.0, 0.0), (40.0, 40.0))),    # dam break (r <= 15)
    (6, 2, ((-3.0, -1.5), (3.0, 2.5))),    # wave towards the bump
])
def test_fill_reference_cases(gpu, ic, bathy, dom):
    c = dict(nx=40, ny=36, x0=dom[0], x1=dom[1], g=9.81, cfl=0.4, bathy_flag=bathy,
             bathy_par=(0.0,) * 5, well_balanced=0)
    s, o = _solver(gpu, c), _oracle(c)
    s.fill_ic(ic)
    o.fill_ic(ic)
    got, ref = s.get_planes(), o.get_planes()
    assert np.all(np.isfinite(got))
    err = _close(got, ref)
    assert err <= RTOL, (ic, err)


def test_unknown_ic_is_an_error(gpu):
    c = cases.case("vortex", n=16)
    s = _solver(gpu, c)
    with pytest.raises(gpu.SwmError):
        s.fill_ic(7)
    with pytest.raises(gpu.SwmError):
        s.fill_ic(101, [0.0] * 9)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_device_wb_lake_at_rest(gpu, precision):
    # WB state and initial state both from the device: U(t) == U(0) exactly
    c = cases.case("lake", n=64)
    s = _solver(gpu, c, precision)
    s.init_wb_ic(c["wb_ic"], c["wb_par"])
    s.fill_ic(c["wb_ic"], c["wb_par"])
    U0 = s.get_planes().copy()
    for _ in range(3):
        s.step(0.0, s.timestep())
    assert np.array_equal(s.get_planes(), U0)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_device_wb_matches_host_wb(gpu, precision):
    # InitializeWBVariables on the device equals swm_set_wb_state of the same cell
    # averages: pulse runs from both are bit-identical.  (A WB state that differs in
    # the last bit -- host libm instead of CUDA's -- moves this pulse run by ~1e-9
    # within three steps: the scheme itself amplifies it, so host and device ICs are
    # compared directly in the fill tests instead.)
    c = cases.case("lake", n=48)
    s_ic = _solver(gpu, c, precision)
    s_ic.fill_ic(c["wb_ic"], c["wb_par"])
    wb = s_ic.get_planes()
    s_dev, s_host = _solver(gpu, c, precision), _solver(gpu, c, precision)
    s_dev.init_wb_ic(c["wb_ic"], c["wb_par"])
    s_host.set_wb_state(cases.ghosted(wb))
    pulse = cases.cell_averages(c)
    s_dev.set_planes(pulse)
    s_host.set_planes(pulse)
    for _ in range(3):
        dt = s_host.timestep()
        s_host.step(0.0, dt)
        s_dev.step(0.0, dt)
    assert np.array_equal(s_dev.get_planes(), s_host.get_planes())


def test_l1_error_matches_oracle(gpu):
    # reference vortex (IC 1) on [0,4]^2: run both to t, compare PostProcessing's L1
    c = dict(nx=40, ny=40, x0=(0.0, 0.0), x1=(4.0, 4.0), g=9.81, cfl=0.4, bathy_flag=0,
             bathy_par=(0.0,) * 5, well_balanced=0)
    s, o = _solver(gpu, c), _oracle(c)
    o.fill_ic(1)
    s.set_planes(o.get_planes())          # identical start: the steps are bitwise equal
    t = 0.0
    for _ in range(4):
        dt = o.timestep()
        assert s.timestep() == dt
        o.step(t, dt)
        s.step(t, dt)
        t += dt
    assert np.array_equal(s.get_planes(), o.get_planes())
    got, ref = s.l1_error(1, t=t), o.l1_error(1, t=t)
    assert np.all(ref > 0)
    assert np.max(np.abs(got - ref) / ref) <= 1e-12, (got, ref)
    # at t = 0 on the device-filled state the error is zero up to the IC rounding
    s.fill_ic(1)
    assert np.all(s.l1_error(1, t=0.0) <= 1e-14)
