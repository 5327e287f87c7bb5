"""Failure paths of the C ABI that a test can reach without faulting a GPU.

* A grid-barrier wait that runs out: the handle's spin limit is set to 0, so every
  Jacobi barrier wait that is not already open gives up at once; the call must
  answer SWM_ERR_WATCHDOG and the next call on the same handle must be bit for bit
  the oracle's again (the control block is cleared before every solve).
* An allocation that fails: the library's own allocator is told to refuse its nth
  allocation; swm_create must answer SWM_ERR_ALLOC and release everything it took.
* A non-finite value born inside a step: the step itself reports SWM_ERR_NAN
  (the reference's mPEuler read of hp(2,nx,ny) through Up(:,1,:,:) produces one,
  timediscretization.f90:734,743,784).
"""
import numpy as np
import pytest

import cases
import oracle as O
from test_gpu_parity import make_pair, random_patankar_system

pytestmark = pytest.mark.gpu

WATCHDOG, ALLOC, NAN = -4, -5, -3


@pytest.mark.parametrize("solver,block", [("stencil", 4), ("csr", 0)])
def test_jacobi_watchdog_then_recovery(gpu, solver, block):
    n = 256  # 64 stencil tiles / 256 CSR blocks: many CTAs wait at every barrier
    c, o, s = make_pair(gpu, "vortex", n, solver=solver, block=block)
    mass, diag, rhs = random_patankar_system(n * n, 7)
    s.set_spin_limit(0)
    with pytest.raises(gpu.SwmError) as e:
        s.debug_jacobi(mass, diag, rhs)
    assert e.value.code == WATCHDOG
    s.set_spin_limit(1 << 26)
    ref, k_ref = o.jacobi(mass, diag, rhs)
    got, k, rc = s.debug_jacobi(mass, diag, rhs)
    assert k == k_ref and rc == 0
    assert np.array_equal(got, ref)


def test_step_watchdog_then_recovery(gpu):
    c, o, s = make_pair(gpu, "island", 128, precision="split", solver="stencil", block=4)
    P0 = s.get_planes().copy()
    dt = s.timestep()
    s.set_spin_limit(0)
    with pytest.raises(gpu.SwmError) as e:
        s.step(0.0, dt)
    assert e.value.code == WATCHDOG
    s.set_spin_limit(1 << 26)
    s.set_planes(P0)
    assert s.timestep() == dt
    assert s.step(0.0, dt) == 0
    # a fresh handle takes the same step
    c2, o2, s2 = make_pair(gpu, "island", 128, precision="split", solver="stencil", block=4)
    s2.step(0.0, s2.timestep())
    assert np.array_equal(s.get_planes(), s2.get_planes())
    assert s.stats()["jacobi_iters"] == s2.stats()["jacobi_iters"]


def test_injected_allocation_failure_releases_everything(gpu):
    import torch
    kw = dict(nx=512, ny=512, x0=(0.0, 0.0), x1=(1.0, 1.0), precision="split",
              solver="stencil", jacobi_block=4, bathy_flag=3, bathy_par=(0.5, 2.0, 0.5, 2.0, 0.5),
              well_balanced=1)
    gpu.inject_alloc_failure(0)
    s = gpu.Solver(**kw)
    s.close()
    total = gpu.inject_alloc_failure(0)  # allocations one swm_create makes
    assert total > 10
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    try:
        for nth in sorted({1, 2, 3, total // 2, total - 2, total - 1, total}):
            gpu.inject_alloc_failure(nth)
            with pytest.raises(gpu.SwmError) as e:
                gpu.Solver(**kw)
            assert e.value.code == ALLOC, nth
            gpu.inject_alloc_failure(0)
            # a leaked plane of this grid would be 2 MiB
            assert abs(torch.cuda.mem_get_info()[0] - free0) < (1 << 20), nth
    finally:
        gpu.inject_alloc_failure(0)
    s = gpu.Solver(**kw)  # the allocator works again
    s.close()


def test_step_reports_nan_born_inside_the_step(gpu):
    # mPEuler with the reference's hp read empties cells to h = 0 in its first step
    # and turns them non-finite in the second
    c, o, s = make_pair(gpu, "dambreak", 32, solver="csr", timescheme=6, compat=1)
    dt = o.timestep()
    assert s.timestep() == dt
    o.step(0.0, dt)
    assert s.step(0.0, dt) == 0
    assert np.array_equal(s.get_planes(), o.get_planes())
    dt = o.timestep()
    assert s.timestep() == dt  # from the reduction that ended the step
    o.step(0.0, dt)
    ref = o.get_planes()
    assert not np.all(np.isfinite(ref))
    with pytest.raises(gpu.SwmError) as e:
        s.step(0.0, dt)
    assert e.value.code == NAN
    assert np.array_equal(s.get_planes(), ref, equal_nan=True)


@pytest.mark.parametrize("per_phase", [False, True])
def test_batch_watchdog_then_recovery(gpu, per_phase):
    # the ensemble's barrier waits give up at once: the step reports the watchdog, and
    # after the limit is restored the same handle steps the restored state exactly as
    # a fresh batch does
    from test_gpu_batch import members, params
    ms = members()[:3]
    P = [cases.cell_averages(c) for c in ms]

    def batch():
        b = gpu.Batch([params(gpu, c, "split", 4) for c in ms])
        b.set_launches(per_phase)
        for i in range(len(ms)):
            b.set_planes(i, P[i])
        return b

    b = batch()
    b.set_spin_limit(0)
    with pytest.raises(gpu.SwmError) as e:
        b.step()
    assert e.value.code == WATCHDOG
    b.set_spin_limit(1 << 26)
    for i in range(len(ms)):
        b.set_planes(i, P[i])
    dts, rc = b.step()
    assert rc == 0
    ref = batch()
    dts_ref, _ = ref.step()
    assert np.array_equal(dts, dts_ref)
    for i in range(len(ms)):
        assert np.array_equal(b.get_planes(i), ref.get_planes(i)), i
    b.close()
    ref.close()
