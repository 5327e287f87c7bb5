"""The other time schemes of timediscretization.f90 on the same RHS kernel, against
the oracle: forward Euler (1), SSPRK(5,4) (2), RK65 (3), DeC5 (4) -- explicit, with
Ut(1) from the mass fluxes as the reference computes it without -DPATANKAR -- and
the modified Patankar Euler (6).  The FP64 form matches bit for bit."""
import numpy as np
import pytest

from test_gpu_parity import make_pair, rel_l1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ts", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("name,n", [("vortex", 40), ("lake", 48)])
def test_scheme_fp64_bitwise(gpu, ts, name, n):
    c, o, s = make_pair(gpu, name, n, precision="fp64", solver="stencil", block=4,
                        timescheme=ts)
    t = 0.0
    for _ in range(3):
        dt = o.timestep()
        assert s.timestep() == dt
        o.step(t, dt)
        s.step(t, dt)
        t += dt
    assert np.array_equal(s.get_planes(), o.get_planes()), ts
    assert s.stats()["n_solves"] == (1 if ts == 6 else 0)


@pytest.mark.parametrize("ts", [2, 4])
def test_scheme_split_close(gpu, ts):
    c, o, s = make_pair(gpu, "vortex", 40, precision="split", solver="stencil", block=4,
                        timescheme=ts)
    for _ in range(3):
        dt = o.timestep()
        o.step(0.0, dt)
        s.step(0.0, dt)
    assert max(rel_l1(s.get_planes(), o.get_planes())) <= 1e-6


def test_mpeuler_compat_and_csr(gpu):
    for compat in (0, 1):
        c, o, s = make_pair(gpu, "dambreak", 32, precision="fp64", solver="csr", timescheme=6,
                            compat=compat)
        for _ in range(2):
            dt = o.timestep()
            o.step(0.0, dt)
            ref = o.get_planes()
            try:
                rc = s.step(0.0, dt)
            except gpu.SwmError as e:  # the step reports non-finite cells it produced
                rc = e.code
            assert rc == (0 if np.all(np.isfinite(ref)) else -3), compat
            if not np.all(np.isfinite(ref)):
                break
        assert np.array_equal(s.get_planes(), o.get_planes(), equal_nan=True), compat
