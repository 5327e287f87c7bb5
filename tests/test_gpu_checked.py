"""The checked build (libswm_checked.so, -DSWM_CHECKED): every wrapped-index site of
the kernels checks its index and records a failure instead of touching memory out of
range.  Small, odd and sub-tile grids, both Jacobi solvers, the mPDeC2 compatibility
read and an ensemble of odd sizes run through it; every check must pass and the FP64
form must still match the oracle bit for bit.  The run is a child process, so that the
checked library is the only one it loads."""
import json
import multiprocessing as mp
import os
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _child(q):
    try:
        sys.path.insert(0, os.path.join(ROOT, "sw-mpdec_b200"))
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np
        import build
        import cases
        import oracle as O
        import swm
        swm.LIB_PATH = build.build(checked=True)
        out = {"runs": 0}
        grids = [("vortex", 5, 7), ("dambreak", 23, 19), ("island", 66, 30), ("lake", 97, 41),
                 ("vortex", 130, 72)]
        for name, nx, ny in grids:
            c = cases.case(name, n=nx)
            c["ny"] = ny
            c["well_balanced"] = 0
            P = cases.cell_averages(c)
            for solver, scheme, compat in (("stencil", 5, 0), ("csr", 5, 0), ("stencil", 7, 1)):
                o = O.Oracle(O.make_params(nx, ny, c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                                           bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                                           timescheme=scheme, mpdec2_compat=compat))
                o.set_planes(P)
                s = swm.Solver(nx=nx, ny=ny, x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                               bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                               timescheme=scheme, mpdec2_compat=compat, precision="fp64",
                               solver=solver, jacobi_block=4)
                s.set_planes(P)
                for _ in range(2):
                    dt = o.timestep()
                    o.step(0.0, dt)
                    try:
                        s.step(0.0, dt)
                    except swm.SwmError as e:  # the compatibility read may produce NaN
                        if e.code != -3:
                            raise
                if not np.array_equal(s.get_planes(), o.get_planes(), equal_nan=True):
                    out["mismatch"] = [name, nx, ny, solver, scheme]
                s.close()
                out["runs"] += 1
            sp = swm.Solver(nx=nx, ny=ny, x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                            bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                            precision="split", solver="stencil", jacobi_block=4)
            sp.set_planes(P)
            sp.step(0.0, sp.timestep())
            sp.close()
        ms = []
        for name, n in (("vortex", 41), ("dambreak", 65), ("island", 33), ("lake", 71)):
            c = cases.case(name, n=n)
            c["well_balanced"] = 0
            ms.append(c)
        for per_phase in (False, True):
            b = swm.Batch([swm.make_params(m["nx"], m["ny"], m["x0"], m["x1"], g=m["g"],
                                           cfl=m["cfl"], bathy_flag=m["bathy_flag"],
                                           bathy_par=m["bathy_par"], precision="split",
                                           solver="stencil", jacobi_block=4) for m in ms])
            b.set_launches(per_phase)
            for i, m in enumerate(ms):
                b.set_planes(i, cases.cell_averages(m))
            b.step()
            b.step()
            b.close()
        out["status"] = swm.checked_status()
        q.put(json.dumps(out))
    except Exception as exc:  # reported to the parent
        q.put(json.dumps({"error": repr(exc)}))


def test_checked_build_records_no_out_of_range_index(gpu):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(q,))
    p.start()
    res = json.loads(q.get(timeout=900))
    p.join(timeout=60)
    assert "error" not in res, res
    assert "mismatch" not in res, res
    assert res["runs"] == 15
    assert res["status"] == [0, 0], res
