"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, always as the checker or the timed CPU restatement, never as part
of the product path.  The C source (swm_oracle.c) restates the reference's
Fortran routines; see its header for the file:line map and the pinning note.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("x0", ctypes.c_double * 2), ("x1", ctypes.c_double * 2),
        ("g", ctypes.c_double), ("cfl", ctypes.c_double),
        ("timescheme", ctypes.c_int), ("bathy_flag", ctypes.c_int),
        ("bathy_par", ctypes.c_double * 5), ("well_balanced", ctypes.c_int),
        ("jacobi_maxiter", ctypes.c_int), ("jacobi_tol", ctypes.c_double),
        ("mpdec2_compat", ctypes.c_int),
    ]


def build():
    """Compile the oracle libraries in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(threaded=False):
    name = "liboracle_omp.so" if threaded else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [P(OrcParams)]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_fill_ic.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    lib.orc_init_wb.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    lib.orc_init_wb_planes.argtypes = [ctypes.c_void_p, dp]
    lib.orc_l1_error.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, ctypes.c_double, dp]
    lib.orc_set_state.argtypes = [ctypes.c_void_p, dp]
    lib.orc_get_state.argtypes = [ctypes.c_void_p, dp, dp]
    lib.orc_get_planes.argtypes = [ctypes.c_void_p, dp]
    lib.orc_set_planes.argtypes = [ctypes.c_void_p, dp]
    lib.orc_timestep.restype = ctypes.c_double
    lib.orc_timestep.argtypes = [ctypes.c_void_p]
    lib.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    lib.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, dp]
    lib.orc_rhs.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp]
    lib.orc_jacobi.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
    lib.orc_rowstart.restype = P(ctypes.c_int)
    lib.orc_rowstart.argtypes = [ctypes.c_void_p]
    lib.orc_columns.restype = P(ctypes.c_int)
    lib.orc_columns.argtypes = [ctypes.c_void_p]
    lib.orc_last_jacobi_iters.argtypes = [ctypes.c_void_p, P(ctypes.c_int), ctypes.c_int]
    lib.orc_total_jacobi_iters.restype = ctypes.c_longlong
    lib.orc_total_jacobi_iters.argtypes = [ctypes.c_void_p]
    lib.orc_mesh_dx.restype = ctypes.c_double
    lib.orc_mesh_dx.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_weno5_first.argtypes = [dp, dp, dp]
    lib.orc_weno5_second.argtypes = [dp, dp]
    lib.orc_quadrature.argtypes = [dp, dp]
    lib.orc_theta_mpdec5.argtypes = [dp, dp]
    lib.orc_patankar_div.restype = ctypes.c_double
    lib.orc_patankar_div.argtypes = [ctypes.c_double, ctypes.c_double]
    lib.orc_bathymetry.argtypes = [P(OrcParams), ctypes.c_double, ctypes.c_double, dp, dp, dp]
    lib.orc_threads.restype = ctypes.c_int
    _LIBS[name] = lib
    return lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(nx, ny, x0, x1, g=9.81, cfl=0.4, timescheme=5, bathy_flag=0,
                bathy_par=(0, 0, 0, 0, 0), well_balanced=0, jacobi_maxiter=1000,
                jacobi_tol=1e-16, mpdec2_compat=0):
    p = OrcParams()
    p.nx, p.ny = nx, ny
    p.x0[0], p.x0[1] = x0
    p.x1[0], p.x1[1] = x1
    p.g, p.cfl = g, cfl
    p.timescheme, p.bathy_flag = timescheme, bathy_flag
    for k in range(5):
        p.bathy_par[k] = bathy_par[k]
    p.well_balanced = well_balanced
    p.jacobi_maxiter, p.jacobi_tol = jacobi_maxiter, jacobi_tol
    p.mpdec2_compat = mpdec2_compat
    return p


class Oracle:
    """One oracle instance: the reference's module state for one grid."""

    def __init__(self, params, threaded=False):
        self.lib = _lib(threaded)
        self.params = params
        self.nx, self.ny = params.nx, params.ny
        self.h = self.lib.orc_create(ctypes.byref(params))
        if not self.h:
            raise ValueError("orc_create failed (nx, ny >= 3 required)")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def ghosted_shape(self):
        return (self.ny + 6, self.nx + 6, 3)

    def fill_ic(self, ic, par=()):
        par = np.ascontiguousarray(np.array(list(par) + [0.0] * 8, dtype=np.float64))
        if self.lib.orc_fill_ic(self.h, ic, _dp(par)) != 0:
            raise ValueError(f"unknown initial condition {ic}")

    def init_wb(self, ic, par=()):
        par = np.ascontiguousarray(np.array(list(par) + [0.0] * 8, dtype=np.float64))
        if self.lib.orc_init_wb(self.h, ic, _dp(par)) != 0:
            raise ValueError(f"unknown WB condition {ic}")

    def l1_error(self, ic, par=(), t=0.0):
        """PostProcessing (postprocessing.f90:23-60): per-variable L1 error of the state
        against the exact solution of `ic` at time t, times dx dy."""
        par = np.ascontiguousarray(np.array(list(par) + [0.0] * 8, dtype=np.float64))
        out = np.zeros(3)
        if self.lib.orc_l1_error(self.h, ic, _dp(par), float(t), _dp(out)) != 0:
            raise ValueError(f"unknown initial condition {ic}")
        return out

    def init_wb_planes(self, planes):
        planes = np.ascontiguousarray(planes, dtype=np.float64)
        assert planes.shape == (3, self.ny, self.nx)
        self.lib.orc_init_wb_planes(self.h, _dp(planes))

    def get_state(self):
        U = np.zeros(self.ghosted_shape)
        V = np.zeros(self.ghosted_shape)
        self.lib.orc_get_state(self.h, _dp(U), _dp(V))
        return U, V

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == self.ghosted_shape
        self.lib.orc_set_state(self.h, _dp(U))

    def get_planes(self):
        out = np.zeros((3, self.ny, self.nx))
        self.lib.orc_get_planes(self.h, _dp(out))
        return out

    def set_planes(self, planes):
        planes = np.ascontiguousarray(planes, dtype=np.float64)
        assert planes.shape == (3, self.ny, self.nx)
        self.lib.orc_set_planes(self.h, _dp(planes))

    def timestep(self):
        return self.lib.orc_timestep(self.h)

    def step(self, t, dt):
        return self.lib.orc_step(self.h, t, dt)

    def run(self, tend, n_outputs=4):
        t = ctypes.c_double(0.0)
        steps = self.lib.orc_run(self.h, tend, n_outputs, ctypes.byref(t))
        return steps, t.value

    def rhs(self):
        nx, ny = self.nx, self.ny
        Ut = np.zeros((ny, nx, 3))
        FX = np.zeros((ny, nx + 1, 3))
        FY = np.zeros((ny + 1, nx, 3))
        S = np.zeros((ny, nx, 3))
        P = np.zeros(5 * nx * ny)
        D = np.zeros(5 * nx * ny)
        self.lib.orc_rhs(self.h, _dp(Ut), _dp(FX), _dp(FY), _dp(S), _dp(P), _dp(D))
        return dict(Ut=Ut, FX=FX, FY=FY, S=S, P=P, D=D)

    def jacobi(self, mass, diag, rhs):
        sol = np.zeros(self.nx * self.ny)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        k = self.lib.orc_jacobi(self.h, _dp(mass), _dp(diag), _dp(rhs), _dp(sol))
        return sol, k

    def csr_pattern(self):
        N = self.nx * self.ny
        rs = np.ctypeslib.as_array(self.lib.orc_rowstart(self.h), shape=(N + 1,)).copy()
        cols = np.ctypeslib.as_array(self.lib.orc_columns(self.h), shape=(5 * N,)).copy()
        return rs, cols

    def last_jacobi_iters(self):
        buf = (ctypes.c_int * 64)()
        n = self.lib.orc_last_jacobi_iters(self.h, buf, 64)
        return list(buf[: min(n, 64)])

    def total_jacobi_iters(self):
        return self.lib.orc_total_jacobi_iters(self.h)

    def dx(self):
        return self.lib.orc_mesh_dx(self.h, 0), self.lib.orc_mesh_dx(self.h, 1)


def weno5_first(q):
    lib = _lib()
    q = np.ascontiguousarray(q, dtype=np.float64)
    wm, wp = ctypes.c_double(), ctypes.c_double()
    lib.orc_weno5_first(_dp(q), ctypes.byref(wm), ctypes.byref(wp))
    return wm.value, wp.value


def weno5_second(q):
    lib = _lib()
    q = np.ascontiguousarray(q, dtype=np.float64)
    w = np.zeros(4)
    lib.orc_weno5_second(_dp(q), _dp(w))
    return w


def quadrature():
    lib = _lib()
    n, w = np.zeros(4), np.zeros(4)
    lib.orc_quadrature(_dp(n), _dp(w))
    return n, w


def bathymetry(params, x, y):
    """Bathymetry b(x, y) of the params (equation.f90:419-450), host libm."""
    b = np.zeros(1)
    _lib().orc_bathymetry(ctypes.byref(params), float(x), float(y), _dp(b), None, None)
    return float(b[0])


def theta_mpdec5():
    lib = _lib()
    th, beta = np.zeros(16), np.zeros(4)
    lib.orc_theta_mpdec5(_dp(th), _dp(beta))
    return th.reshape(4, 4), beta


def patankar_div(p, h):
    return _lib().orc_patankar_div(p, h)


def threads(threaded=True):
    return _lib(threaded).orc_threads()
