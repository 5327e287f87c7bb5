"""swm_jacobi_noalloc: the Jacobi solve for callers that cannot let a library
allocate device memory (drivers that own all device memory through their own
pool or a shared memory cap, loops that cannot afford cudaMalloc/cudaFree's
device-wide synchronisation).  It must give the same answer as the handle
solver (swm_debug_jacobi with the stencil solver) on repeated calls, while its
only scratch is a static device array that keeps the previous call's contents.

This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

import swm


def patankar_system(n_cells, seed):
    """An M-matrix in the reference CSR slot order (S, W, C, E, N), positive rhs."""
    rng = np.random.default_rng(seed)
    mass = -0.1 * rng.random((n_cells, 5))
    mass[:, 2] = 0.0
    diag = 1.0 + 0.4 * rng.random(n_cells)
    rhs = 0.5 + rng.random(n_cells)
    return mass, diag, rhs


def test_noalloc_rejects_grids_beyond_its_scratch():
    # size check happens before any CUDA call
    lib = swm.load()
    it = ctypes.c_int()
    one = ctypes.c_void_p(16)
    rc = lib.swm_jacobi_noalloc(2048, 2048, *([one] * 6), ctypes.c_void_p(32), 1000, 1e-16, 4,
                                ctypes.byref(it), None)
    assert rc == -1
    assert b"1048576" in lib.swm_last_error()


@pytest.mark.parametrize("where", ["rhs", "cS", "cD"])
def test_noalloc_rejects_sol_overlapping_an_input(where):
    # sol is written while the inputs are read: a view one double into rhs or a
    # coefficient plane is refused before any CUDA call (the addresses are never
    # dereferenced)
    lib = swm.load()
    nx, ny = 16, 16
    nbytes = nx * ny * 8
    base = {"cS": 1 << 20, "cW": 2 << 20, "cE": 3 << 20, "cN": 4 << 20, "cD": 5 << 20,
            "rhs": 6 << 20}
    sol = base[where] + 8 if where != "cD" else base[where] - nbytes + 8
    ptrs = [ctypes.c_void_p(base[k]) for k in ("cS", "cW", "cE", "cN", "cD", "rhs")]
    it = ctypes.c_int()
    rc = lib.swm_jacobi_noalloc(nx, ny, *ptrs, ctypes.c_void_p(sol), 1000, 1e-16, 4,
                                ctypes.byref(it), None)
    assert rc == -1
    assert b"overlap" in lib.swm_last_error()


def device_system(torch, dev, mass, diag, rhs):
    planes = [torch.from_numpy(np.ascontiguousarray(mass[:, k])).to(dev) for k in (0, 1, 3, 4)]
    return planes + [torch.from_numpy(diag).to(dev), torch.from_numpy(rhs).to(dev)]


@pytest.mark.gpu
def test_noalloc_matches_handle_solver_twice(gpu):
    import torch
    nx, ny, block = 96, 80, 4
    N = nx * ny
    s = swm.Solver(nx=nx, ny=ny, x0=(0.0, 0.0), x1=(1.0, 1.0), solver="stencil",
                   jacobi_block=block)
    dev = torch.device("cuda", 0)
    for call, seed in enumerate((11, 12)):
        mass, diag, rhs = patankar_system(N, seed)
        ref, k_ref, rc_ref = s.debug_jacobi(mass.reshape(-1), diag, rhs)
        planes = [torch.from_numpy(np.ascontiguousarray(mass[:, k])).to(dev)
                  for k in (0, 1, 3, 4)]
        cD = torch.from_numpy(diag).to(dev)
        b = torch.from_numpy(rhs).to(dev)
        sol = torch.full((N,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        k, rc = swm.jacobi_noalloc(nx, ny, *[p.data_ptr() for p in planes], cD.data_ptr(),
                                   b.data_ptr(), sol.data_ptr(), block=block)
        assert (k, rc) == (k_ref, rc_ref), call
        assert np.array_equal(sol.cpu().numpy(), ref), call
    s.close()


@pytest.mark.gpu
def test_noalloc_arrays_off_16_byte_boundaries(gpu):
    # Caller arrays that start 8 bytes past a 16-byte boundary (views one double into
    # a larger buffer): the solve must take its 8-byte copy path and still agree
    # with the handle solver bit for bit.
    import torch
    nx, ny, block = 96, 80, 4
    N = nx * ny
    s = swm.Solver(nx=nx, ny=ny, x0=(0.0, 0.0), x1=(1.0, 1.0), solver="stencil",
                   jacobi_block=block)
    dev = torch.device("cuda", 0)
    mass, diag, rhs = patankar_system(N, 21)
    ref, k_ref, rc_ref = s.debug_jacobi(mass.reshape(-1), diag, rhs)

    def offset_view(host):
        buf = torch.zeros(N + 1, dtype=torch.float64, device=dev)
        buf[1:] = torch.from_numpy(np.ascontiguousarray(host)).to(dev)
        view = buf[1:]
        assert view.data_ptr() % 16 == 8
        return buf, view

    keep = [offset_view(mass[:, k]) for k in (0, 1, 3, 4)]
    keep += [offset_view(diag), offset_view(rhs), offset_view(np.full(N, np.nan))]
    views = [v for _, v in keep]
    torch.cuda.synchronize()
    k, rc = swm.jacobi_noalloc(nx, ny, *[v.data_ptr() for v in views], block=block)
    assert (k, rc) == (k_ref, rc_ref)
    assert np.array_equal(views[-1].cpu().numpy(), ref)
    s.close()


@pytest.mark.gpu
def test_noalloc_maxiter_warning_matches_handle_solver(gpu):
    # a solve cut off at maxiter: warning 1 and the same iterate as the handle solver
    import torch
    nx, ny, block = 64, 48, 2
    N = nx * ny
    s = swm.Solver(nx=nx, ny=ny, x0=(0.0, 0.0), x1=(1.0, 1.0), solver="stencil",
                   jacobi_block=block, jacobi_maxiter=3)
    dev = torch.device("cuda", 0)
    mass, diag, rhs = patankar_system(N, 31)
    ref, k_ref, rc_ref = s.debug_jacobi(mass.reshape(-1), diag, rhs)
    assert (k_ref, rc_ref) == (3, 1)
    arrs = device_system(torch, dev, mass, diag, rhs)
    sol = torch.full((N,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    k, rc = swm.jacobi_noalloc(nx, ny, *[a.data_ptr() for a in arrs], sol.data_ptr(),
                               maxiter=3, block=block)
    assert (k, rc) == (3, 1)
    assert np.array_equal(sol.cpu().numpy(), ref)
    s.close()


@pytest.mark.gpu
def test_noalloc_on_a_caller_stream_at_the_cell_limit(gpu):
    # 1024 x 1024 fills the static iterate buffer up to the control block; the solve
    # runs on a stream the caller created; a second call changes no device memory use
    import torch
    nx = ny = 1024
    N = nx * ny
    block = 4
    s = swm.Solver(nx=nx, ny=ny, x0=(0.0, 0.0), x1=(1.0, 1.0), solver="stencil",
                   jacobi_block=block)
    dev = torch.device("cuda", 0)
    mass, diag, rhs = patankar_system(N, 41)
    ref, k_ref, rc_ref = s.debug_jacobi(mass.reshape(-1), diag, rhs)
    arrs = device_system(torch, dev, mass, diag, rhs)
    sol = torch.full((N,), float("nan"), dtype=torch.float64, device=dev)
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    k, rc = swm.jacobi_noalloc(nx, ny, *[a.data_ptr() for a in arrs], sol.data_ptr(),
                               block=block, stream=st.cuda_stream)
    assert (k, rc) == (k_ref, rc_ref)
    assert np.array_equal(sol.cpu().numpy(), ref)
    free_before = torch.cuda.mem_get_info()[0]
    sol.fill_(float("nan"))
    torch.cuda.synchronize()
    k2, rc2 = swm.jacobi_noalloc(nx, ny, *[a.data_ptr() for a in arrs], sol.data_ptr(),
                                 block=block, stream=st.cuda_stream)
    assert torch.cuda.mem_get_info()[0] == free_before
    assert (k2, rc2) == (k_ref, rc_ref)
    assert np.array_equal(sol.cpu().numpy(), ref)
    s.close()


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream(gpu):
    # the call synchronises its stream to read the iteration count, which a stream
    # under capture cannot do: it answers SWM_ERR_STATE without enqueuing anything
    import torch
    nx, ny = 32, 32
    N = nx * ny
    dev = torch.device("cuda", 0)
    mass, diag, rhs = patankar_system(N, 51)
    arrs = device_system(torch, dev, mass, diag, rhs)
    sol = torch.zeros(N, dtype=torch.float64, device=dev)
    lib = swm.load()
    it = ctypes.c_int()
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(st):
        g.capture_begin()
        rc = lib.swm_jacobi_noalloc(nx, ny, *[ctypes.c_void_p(a.data_ptr()) for a in arrs],
                                    ctypes.c_void_p(sol.data_ptr()), 1000, 1e-16, 4,
                                    ctypes.byref(it), ctypes.c_void_p(st.cuda_stream))
        sol.add_(1.0)  # the capture stays valid: give it one node
        g.capture_end()
    assert rc == -6
    assert b"capture" in lib.swm_last_error()
