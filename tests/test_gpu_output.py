"""Device-formatted solution output (swm_write_output / swm_write_mesh /
swm_debug_format) against the CPU restatement of output.f90 (oracle/output.py)."""
import math
import os

import numpy as np
import pytest

import cases
import oracle as O
import output as OUT

pytestmark = pytest.mark.gpu


def _solver(swm, c, **kw):
    return swm.Solver(nx=c["nx"], ny=c["ny"], x0=c["x0"], x1=c["x1"], g=c["g"], cfl=c["cfl"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                      precision="fp64", solver="stencil", jacobi_block=4, **kw)


def test_formatter_matches_correct_rounding(gpu):
    c = cases.case("vortex", n=16)
    s = _solver(gpu, c)
    edge = [0.0, -0.0, 1.0, -1.0, 0.1, 1.0 / 3.0, 2.0 / 3.0, 1e-70, -1e-70, 9.9999999999999995,
            1.0 + 2.0**-15, 1.0 + 3 * 2.0**-15, 123456789012345.5, 0.5, 1e99, 9.99999999999999e99,
            1e100, 1e-99, 1e-100, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
            float("nan"), float("inf"), float("-inf"), 1e-6, 9.81, 4.0 / 2048.0]
    rng = np.random.default_rng(7)
    mant = rng.random(20000) * 9.0 + 1.0
    expo = rng.integers(-99, 100, 20000).astype(float)
    rnd = mant * 10.0**expo * np.where(rng.random(20000) < 0.5, -1.0, 1.0)
    bits = rng.integers(0, 2**63, 20000, dtype=np.uint64).view(np.float64)   # any finite double
    vals = np.concatenate([np.array(edge), rnd, bits[np.isfinite(bits)]])
    got = s.format_values(vals)
    bad = [(v, g, OUT.es21(v)) for v, g in zip(vals, got) if g != OUT.es21(v)]
    assert not bad, bad[:5]


def _read(path):
    with open(path) as f:
        return f.read()


@pytest.mark.parametrize("which", [2, 1, 3])
def test_write_output_files(gpu, tmp_path, which):
    # reference vortex (IC 1) on [0,4]^2, a few mPDeC5 steps, then WriteSolutionToDisk(t)
    c = dict(nx=24, ny=16, x0=(0.0, 0.0), x1=(4.0, 4.0), g=9.81, cfl=0.4, bathy_flag=0,
             bathy_par=(0.0,) * 5)
    s = _solver(gpu, c)
    s.fill_ic(1)
    t = 0.0
    for _ in range(2):
        dt = s.timestep()
        s.step(t, dt)
        t += dt
    s.write_output(t, str(tmp_path), which_output=which, ic=1)
    P = s.get_planes()
    V = OUT.cons_to_prim(P)                          # IEEE quotients, as the device rounds
    bath = np.zeros_like(P[0])   # flat bottom
    names = []
    if which in (2, 3):
        names += [("SOLUTION_TEC", "tec"), ("ERROR_TEC", "tec")]
    if which in (1, 3):
        names += [("SOLUTION_OCT", "oct"), ("ERROR_OCT", "oct")]
    assert sorted(os.listdir(tmp_path)) == sorted(OUT.timestamp(n, t) + ".dat" for n, _ in names)
    for name, kind in names:
        txt = _read(tmp_path / (OUT.timestamp(name, t) + ".dat"))
        if name.startswith("SOLUTION"):
            planes = [V[0], V[1], V[2], bath]
            want = (OUT.tecplot_text(t, c["nx"], c["ny"], c["x0"], c["x1"], planes)
                    if kind == "tec" else OUT.octave_text(planes))
            assert txt == want, name       # byte for byte (bathymetry flat: Bath = 0)
        else:
            lines = txt.splitlines()
            hdr = 2 if kind == "tec" else 1
            want = (OUT.tecplot_text(t, c["nx"], c["ny"], c["x0"], c["x1"],
                                     [P[0], P[1], P[2], bath])
                    if kind == "tec" else OUT.octave_text([P[0], P[1], P[2], bath]))
            assert lines[:hdr] == want.splitlines()[:hdr]
            vals = np.array([[float(v) for v in ln.split()] for ln in lines[hdr:]])
            err = vals[:, -4:-1].reshape(c["ny"], c["nx"], 3)
            # |U - Uexact(t)| is the scheme's error: small and consistent with the L1 error
            l1 = s.l1_error(1, t=t)
            dxdy = (4.0 / c["nx"]) * (4.0 / c["ny"])
            for v in range(3):
                assert abs(np.abs(err[..., v]).sum() * dxdy - l1[v]) <= 1e-12 + 1e-9 * l1[v]
            assert np.all(vals[:, -1] == 0.0)


def test_write_mesh_and_bathymetry(gpu, tmp_path):
    c = cases.case("island", n=32)
    s = _solver(gpu, c)
    s.fill_ic(c["ic"], c["par"])
    s.write_mesh(str(tmp_path))
    for d, f in ((0, "MESH_CoordinateX.dat"), (1, "MESH_CoordinateY.dat")):
        assert _read(tmp_path / f) == OUT.mesh_text(c["nx"], c["ny"], c["x0"], c["x1"], d)
    s.write_output(0.0, str(tmp_path), which_output=2, ic=c["ic"], par=c["par"])
    txt = _read(tmp_path / (OUT.timestamp("SOLUTION_TEC", 0.0) + ".dat")).splitlines()
    vals = np.array([[float(v) for v in ln.split()] for ln in txt[2:]])
    # Bath: 4x4 Gauss average of b (finitevolume.f90:323-325), CUDA's exp vs the host's
    prm = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], bathy_flag=c["bathy_flag"],
                        bathy_par=c["bathy_par"])
    qn, qw = O.quadrature()
    X, Y = OUT.barycentres(c["nx"], c["ny"], c["x0"], c["x1"])
    dx, dy = (c["x1"][0] - c["x0"][0]) / c["nx"], (c["x1"][1] - c["x0"][1]) / c["ny"]
    bath = np.zeros((c["ny"], c["nx"]))
    for a in range(4):
        for b in range(4):
            bath += qw[a] * qw[b] * np.vectorize(lambda x, y: O.bathymetry(prm, x, y))(
                X + qn[a] * dx, Y + qn[b] * dy)
    bath[np.abs(bath) < 1e-70] = 0.0
    assert np.allclose(vals[:, 5], bath.ravel(), rtol=1e-13, atol=0)
    assert math.isclose(vals[:, 0].min(), X.min()) and math.isclose(vals[:, 1].max(), Y.max())
