"""ctypes binding of libswm.so (include/swm.h), the sm_100a mPDeC5 time step.

This mirrors the reference's time-step interface for Python callers (tests,
bench): ``Solver.timestep()`` is ``TimeStep()`` (equation.f90:791-837) and
``Solver.step(t, dt)`` is ``TimeDiscretizationByMPDeC5(t)``
(timediscretization.f90:458-566).  There is no CPU fallback: if the library is
missing or no B200 is present, construction raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libswm.so")

OK, WARN_JACOBI_MAXITER = 0, 1
ERR = {-1: "PARAM", -2: "CUDA", -3: "NAN", -4: "WATCHDOG", -5: "ALLOC", -6: "STATE",
       -7: "UNSUPPORTED"}
PREC = {"fp64": 0, "split": 1, "fp64_fma": 2}
SOLVER = {"csr": 0, "stencil": 1}

# Every exported entry point declared in include/swm.h.
EXPORTS = [
    "swm_params_default", "swm_create", "swm_destroy", "swm_set_state", "swm_get_state",
    "swm_set_planes", "swm_get_planes", "swm_set_wb_state", "swm_timestep", "swm_step",
    "swm_run", "swm_get_stats", "swm_state_summary", "swm_last_error", "swm_strerror",
    "swm_get_stream", "swm_profile_step", "swm_debug_rhs", "swm_debug_jacobi", "swm_batch_create", "swm_batch_destroy",
    "swm_batch_set_planes", "swm_batch_get_planes", "swm_batch_step", "swm_batch_cells",
    "swm_jacobi_noalloc", "swm_batch_get_stats", "swm_batch_get_stream",
    "swm_fill_ic", "swm_init_wb_ic", "swm_l1_error", "swm_write_output", "swm_write_mesh",
    "swm_debug_format", "swm_debug_set_spin_limit", "swm_debug_inject_alloc_failure",
    "swm_debug_set_tma", "swm_batch_debug_set_launches", "swm_batch_get_launch_info",
    "swm_batch_debug_phase_times", "swm_batch_debug_set_spin_limit",
    "swm_debug_checked_status",
]


class SwmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"swm error {code} ({ERR.get(code, '?')}): {msg}")
        self.code = code


class SwmParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("x0", ctypes.c_double * 2), ("x1", ctypes.c_double * 2),
        ("g", ctypes.c_double), ("cfl", ctypes.c_double),
        ("timescheme", ctypes.c_int), ("bathy_flag", ctypes.c_int),
        ("bathy_par", ctypes.c_double * 5), ("well_balanced", ctypes.c_int),
        ("precision", ctypes.c_int), ("solver", ctypes.c_int),
        ("jacobi_maxiter", ctypes.c_int), ("jacobi_tol", ctypes.c_double),
        ("jacobi_block", ctypes.c_int), ("mpdec2_compat", ctypes.c_int),
        ("use_graph", ctypes.c_int), ("device", ctypes.c_int),
        ("source_table", ctypes.c_int),
    ]


class SwmStats(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("n_solves", ctypes.c_int),
        ("jacobi_iters", ctypes.c_int * 16),
        ("jacobi_iters_min", ctypes.c_int), ("jacobi_iters_max", ctypes.c_int),
        ("jacobi_iters_total", ctypes.c_longlong), ("steps", ctypes.c_longlong),
        ("lambda_max", ctypes.c_double * 2),
    ]


_lib = None


def load():
    """Load libswm.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built: run `python sw-mpdec_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    vp = ctypes.c_void_p
    lib.swm_params_default.argtypes = [P(SwmParams), ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4
    lib.swm_create.argtypes = [P(SwmParams), P(vp)]
    lib.swm_destroy.argtypes = [vp]
    lib.swm_set_state.argtypes = [vp, dp]
    lib.swm_get_state.argtypes = [vp, dp, dp]
    lib.swm_set_planes.argtypes = [vp, dp]
    lib.swm_get_planes.argtypes = [vp, dp]
    lib.swm_set_wb_state.argtypes = [vp, dp]
    lib.swm_fill_ic.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int]
    lib.swm_init_wb_ic.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int]
    lib.swm_l1_error.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]
    lib.swm_write_output.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp,
                                     ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    lib.swm_write_mesh.argtypes = [vp, ctypes.c_char_p]
    lib.swm_debug_format.argtypes = [vp, dp, ctypes.c_int, ctypes.c_char_p]
    lib.swm_timestep.argtypes = [vp, dp]
    lib.swm_step.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    lib.swm_run.argtypes = [vp, ctypes.c_double, ctypes.c_int, P(ctypes.c_int), dp]
    lib.swm_get_stats.argtypes = [vp, P(SwmStats)]
    lib.swm_state_summary.argtypes = [vp, dp, dp]
    lib.swm_last_error.restype = ctypes.c_char_p
    lib.swm_strerror.restype = ctypes.c_char_p
    lib.swm_strerror.argtypes = [ctypes.c_int]
    lib.swm_get_stream.argtypes = [vp, P(vp)]
    lib.swm_profile_step.argtypes = [vp, ctypes.c_double, ctypes.c_double, P(ctypes.c_float),
                                     P(ctypes.c_int)]
    lib.swm_debug_rhs.argtypes = [vp, dp, dp, dp, dp, dp]
    lib.swm_debug_jacobi.argtypes = [vp, dp, dp, dp, dp, P(ctypes.c_int)]
    lib.swm_debug_set_spin_limit.argtypes = [vp, ctypes.c_longlong]
    lib.swm_debug_set_tma.argtypes = [vp, ctypes.c_int]
    lib.swm_debug_inject_alloc_failure.argtypes = [ctypes.c_longlong, P(ctypes.c_longlong)]
    lib.swm_batch_create.argtypes = [ctypes.c_int, P(SwmParams), P(vp)]
    lib.swm_batch_destroy.argtypes = [vp]
    lib.swm_batch_set_planes.argtypes = [vp, ctypes.c_int, dp]
    lib.swm_batch_get_planes.argtypes = [vp, ctypes.c_int, dp]
    lib.swm_batch_step.argtypes = [vp, dp]
    lib.swm_batch_cells.argtypes = [vp, P(ctypes.c_longlong)]
    lib.swm_batch_get_stats.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_longlong),
                                        P(ctypes.c_int)]
    lib.swm_batch_get_stream.argtypes = [vp, P(vp)]
    lib.swm_batch_debug_set_launches.argtypes = [vp, ctypes.c_int]
    lib.swm_batch_get_launch_info.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int)]
    lib.swm_batch_debug_phase_times.argtypes = [vp, dp, ctypes.c_int, P(ctypes.c_int)]
    lib.swm_batch_debug_set_spin_limit.argtypes = [vp, ctypes.c_longlong]
    lib.swm_debug_checked_status.argtypes = [P(ctypes.c_int), P(ctypes.c_ulonglong)]
    lib.swm_jacobi_noalloc.argtypes = ([ctypes.c_int, ctypes.c_int] + [vp] * 7 +
                                       [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        P(ctypes.c_int), vp])
    _lib = lib
    return lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc):
    if rc < 0:
        raise SwmError(rc, load().swm_last_error().decode())
    return rc


def make_params(nx, ny, x0, x1, g=9.81, cfl=1.0, timescheme=5, bathy_flag=0,
                bathy_par=(0, 0, 0, 0, 0), well_balanced=0, precision="fp64", solver="csr",
                jacobi_maxiter=1000, jacobi_tol=1e-16, jacobi_block=0, mpdec2_compat=0,
                use_graph=1, device=0, source_table=1):
    lib = load()
    p = SwmParams()
    _check(lib.swm_params_default(ctypes.byref(p), nx, ny, x0[0], x0[1], x1[0], x1[1]))
    p.g, p.cfl, p.timescheme, p.bathy_flag = g, cfl, timescheme, bathy_flag
    for k in range(5):
        p.bathy_par[k] = bathy_par[k]
    p.well_balanced = int(well_balanced)
    p.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    p.solver = SOLVER[solver] if isinstance(solver, str) else int(solver)
    p.jacobi_maxiter, p.jacobi_tol, p.jacobi_block = jacobi_maxiter, jacobi_tol, jacobi_block
    p.mpdec2_compat, p.use_graph, p.device = int(mpdec2_compat), int(use_graph), device
    p.source_table = int(source_table)
    return p


class Solver:
    """One grid's device state and time step (a handle of the C ABI)."""

    def __init__(self, params=None, **kw):
        self.lib = load()
        self.params = params if params is not None else make_params(**kw)
        self.nx, self.ny = self.params.nx, self.params.ny
        h = ctypes.c_void_p()
        _check(self.lib.swm_create(ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.swm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def ghosted_shape(self):
        return (self.ny + 6, self.nx + 6, 3)

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == self.ghosted_shape
        _check(self.lib.swm_set_state(self.h, _dp(U)))

    def get_state(self, with_v=False):
        U = np.zeros(self.ghosted_shape)
        V = np.zeros(self.ghosted_shape) if with_v else None
        _check(self.lib.swm_get_state(self.h, _dp(U), _dp(V)))
        return (U, V) if with_v else U

    def set_planes(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        assert P.shape == (3, self.ny, self.nx)
        _check(self.lib.swm_set_planes(self.h, _dp(P)))

    def get_planes(self, out=None):
        P = out if out is not None else np.zeros((3, self.ny, self.nx))
        _check(self.lib.swm_get_planes(self.h, _dp(P)))
        return P

    def set_wb_state(self, Uwb):
        Uwb = np.ascontiguousarray(Uwb, dtype=np.float64)
        _check(self.lib.swm_set_wb_state(self.h, _dp(Uwb)))

    @staticmethod
    def _par(par):
        par = np.ascontiguousarray(np.array(list(par) if par is not None else [], dtype=np.float64))
        return (_dp(par) if par.size else None), int(par.size), par

    def fill_ic(self, ic, par=()):
        """U := 4x4 Gauss averages of ExactFunction case `ic` (FillInitialConditions)."""
        p, n, keep = self._par(par)
        _check(self.lib.swm_fill_ic(self.h, int(ic), p, n))

    def init_wb_ic(self, ic, par=()):
        """InitializeWBVariables from case `ic` evaluated on the device."""
        p, n, keep = self._par(par)
        _check(self.lib.swm_init_wb_ic(self.h, int(ic), p, n))

    def l1_error(self, ic, par=(), t=0.0):
        """PostProcessing: per-variable L1 error against ExactFunction(ic, t), times dx dy."""
        p, n, keep = self._par(par)
        out = np.zeros(3)
        _check(self.lib.swm_l1_error(self.h, int(ic), p, n, float(t), _dp(out)))
        return out

    def write_output(self, t, directory, which_output=2, ic=1, par=(), v_last_rhs=False):
        """WriteSolutionToDisk(t): SOLUTION_* / ERROR_* files in `directory`."""
        p, n, keep = self._par(par)
        _check(self.lib.swm_write_output(self.h, float(t), int(which_output), int(ic), p, n,
                                         os.fsencode(directory), 1 if v_last_rhs else 0))

    def write_mesh(self, directory):
        _check(self.lib.swm_write_mesh(self.h, os.fsencode(directory)))

    def format_values(self, x):
        """(SP,ES21.14E2) strings of the values, formatted on the device."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
        buf = ctypes.create_string_buffer(21 * max(x.size, 1))
        _check(self.lib.swm_debug_format(self.h, _dp(x), int(x.size), buf))
        raw = buf.raw[:21 * x.size].decode()
        return [raw[21 * k:21 * k + 21] for k in range(x.size)]

    def timestep(self):
        dt = ctypes.c_double()
        _check(self.lib.swm_timestep(self.h, ctypes.byref(dt)))
        return dt.value

    def step(self, t, dt):
        return _check(self.lib.swm_step(self.h, t, dt))

    def run(self, t_end, n_outputs=4):
        n = ctypes.c_int()
        t = ctypes.c_double()
        _check(self.lib.swm_run(self.h, t_end, n_outputs, ctypes.byref(n), ctypes.byref(t)))
        return n.value, t.value

    def stats(self):
        s = SwmStats()
        _check(self.lib.swm_get_stats(self.h, ctypes.byref(s)))
        return dict(status=s.status, n_solves=s.n_solves,
                    jacobi_iters=list(s.jacobi_iters[: s.n_solves]),
                    jacobi_iters_min=s.jacobi_iters_min, jacobi_iters_max=s.jacobi_iters_max,
                    jacobi_iters_total=s.jacobi_iters_total, steps=s.steps,
                    lambda_max=(s.lambda_max[0], s.lambda_max[1]))

    def summary(self):
        m, mn = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.swm_state_summary(self.h, ctypes.byref(m), ctypes.byref(mn)))
        return m.value, mn.value

    def stream(self):
        """cudaStream_t of the handle, as an integer (for torch.cuda.ExternalStream)."""
        p = ctypes.c_void_p()
        _check(self.lib.swm_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def profile_step(self, t, dt):
        ms = (ctypes.c_float * 4)()
        n = (ctypes.c_int * 3)()
        _check(self.lib.swm_profile_step(self.h, t, dt, ms, n))
        return dict(rhs_ms=ms[0], assemble_ms=ms[1], jacobi_ms=ms[2], step_ms=ms[3],
                    rhs_launches=n[0], assemble_launches=n[1], jacobi_launches=n[2])

    def debug_rhs(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        nx, ny = self.nx, self.ny
        Ut = np.zeros((ny, nx, 3))
        FX = np.zeros((ny, nx + 1, 3))
        FY = np.zeros((ny + 1, nx, 3))
        S = np.zeros((ny, nx, 3))
        _check(self.lib.swm_debug_rhs(self.h, _dp(U), _dp(Ut), _dp(FX), _dp(FY), _dp(S)))
        return dict(Ut=Ut, FX=FX, FY=FY, S=S)

    def set_tma(self, enable):
        """RHS tile loads by TMA (True, default) or by wrapped-index loads (False)."""
        _check(self.lib.swm_debug_set_tma(self.h, 1 if enable else 0))

    def set_spin_limit(self, limit):
        """Polls of each Jacobi grid-barrier wait before SWM_ERR_WATCHDOG (<= 0: at once)."""
        _check(self.lib.swm_debug_set_spin_limit(self.h, int(limit)))

    def debug_jacobi(self, mass, diag, rhs):
        n = self.nx * self.ny
        sol = np.zeros(n)
        it = ctypes.c_int()
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        rc = _check(self.lib.swm_debug_jacobi(self.h, _dp(mass), _dp(diag), _dp(rhs), _dp(sol),
                                              ctypes.byref(it)))
        return sol, it.value, rc


def checked_status():
    """(site, count) of the checked build's failing index checks, cleared; raises
    SwmError(SWM_ERR_UNSUPPORTED) in the normal build."""
    lib = load()
    site, count = ctypes.c_int(), ctypes.c_ulonglong()
    _check(lib.swm_debug_checked_status(ctypes.byref(site), ctypes.byref(count)))
    return site.value, count.value


def inject_alloc_failure(nth):
    """Make the library's nth allocation from now fail (0: none); returns the number
    of allocations counted since the previous call."""
    n = ctypes.c_longlong()
    _check(load().swm_debug_inject_alloc_failure(int(nth), ctypes.byref(n)))
    return n.value


def jacobi_noalloc(nx, ny, cS, cW, cE, cN, cD, rhs, sol, maxiter=1000, tol=1e-16, block=4,
                   stream=0):
    """swm_jacobi_noalloc: one Patankar Jacobi solve on caller-owned device arrays
    (integer device addresses), with no allocation by the library.  Returns
    (iterations, status)."""
    it = ctypes.c_int()
    ptrs = [ctypes.c_void_p(int(p)) for p in (cS, cW, cE, cN, cD, rhs, sol)]
    rc = _check(load().swm_jacobi_noalloc(nx, ny, *ptrs, maxiter, tol, block, ctypes.byref(it),
                                          ctypes.c_void_p(int(stream))))
    return it.value, rc


class Batch:
    """An ensemble of independent problems stepped together."""

    def __init__(self, params_list):
        self.lib = load()
        arr = (SwmParams * len(params_list))(*params_list)
        self.params = list(params_list)
        h = ctypes.c_void_p()
        _check(self.lib.swm_batch_create(len(params_list), arr, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.swm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_planes(self, i, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        _check(self.lib.swm_batch_set_planes(self.h, i, _dp(P)))

    def get_planes(self, i):
        p = self.params[i]
        P = np.zeros((3, p.ny, p.nx))
        _check(self.lib.swm_batch_get_planes(self.h, i, _dp(P)))
        return P

    def step(self):
        dts = np.zeros(len(self.params))
        rc = _check(self.lib.swm_batch_step(self.h, _dp(dts)))
        return dts, rc

    def cells(self):
        c = ctypes.c_longlong()
        _check(self.lib.swm_batch_cells(self.h, ctypes.byref(c)))
        return c.value

    def stream(self):
        p = ctypes.c_void_p()
        _check(self.lib.swm_batch_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def set_launches(self, per_phase):
        """The step form: a kernel per phase (True; 17 launches per step for the split
        and FMA forms, 25 for FP64), the persistent launch (False), or the autotuner's
        choice (None)."""
        v = -1 if per_phase is None else (1 if per_phase else 0)
        _check(self.lib.swm_batch_debug_set_launches(self.h, v))

    def phase_times(self):
        """Durations (ms) of the step's phases over one step in the current form (which
        advances the state): TimeStep, RHS of U^n, then per correction assembly,
        Jacobi, RHS."""
        ms = np.zeros(32)
        n = ctypes.c_int()
        _check(self.lib.swm_batch_debug_phase_times(self.h, _dp(ms), 32, ctypes.byref(n)))
        names = ["timestep", "rhs_Un"]
        for k in range(1, 6):
            names += [f"assemble_k{k}", f"jacobi_k{k}"] + ([f"rhs_k{k}"] if k < 5 else [])
        return dict(zip(names, ms[: n.value].tolist()))

    def set_spin_limit(self, limit):
        """Polls of each grid-barrier wait before SWM_ERR_WATCHDOG (<= 0: at once)."""
        _check(self.lib.swm_batch_debug_set_spin_limit(self.h, int(limit)))

    def launch_info(self):
        """(kernel launches per step, CTAs of the persistent launch)."""
        n, c = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.swm_batch_get_launch_info(self.h, ctypes.byref(n), ctypes.byref(c)))
        return n.value, c.value

    def stats(self):
        """(sweeps per Jacobi pass, total sweeps, last step's sweeps [13][n])."""
        blk, tot = ctypes.c_int(), ctypes.c_longlong()
        last = np.zeros(13 * len(self.params), dtype=np.int32)
        _check(self.lib.swm_batch_get_stats(self.h, ctypes.byref(blk), ctypes.byref(tot),
                                            last.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return blk.value, tot.value, last.reshape(13, len(self.params))
