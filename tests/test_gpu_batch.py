"""Ensembles (swm_batch_*): every member of a batched step is bit-identical to the
same problem stepped alone with the same precision and solver (the batched
kernels run the single-grid tile code per problem, dt per problem comes from the
same formula on the device), and the autotuner's choice does not change results."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def members():
    out = []
    for name, n in (("vortex", 40), ("dambreak", 56), ("lake", 72), ("island", 50),
                    ("lake_dry", 40)):
        c = cases.case(name, n=n)
        c["well_balanced"] = 0
        out.append(c)
    return out


def params(swm, c, precision, block):
    return swm.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                           bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                           precision=precision, solver="stencil", jacobi_block=block)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_batch_members_match_single_solvers(gpu, precision):
    swm = gpu
    ms = members()
    b = swm.Batch([params(swm, c, precision, 4) for c in ms])
    assert b.cells() == sum(c["nx"] * c["ny"] for c in ms)
    singles = []
    for i, c in enumerate(ms):
        P = cases.cell_averages(c)
        b.set_planes(i, P)
        s = swm.Solver(params(swm, c, precision, 4))
        s.set_planes(P)
        singles.append(s)
    for step in range(2):
        dts, rc = b.step()
        assert rc == 0
        for i, s in enumerate(singles):
            dt = s.timestep()
            assert dt == dts[i]
            s.step(0.0, dt)
    blk, tot, last = b.stats()
    for i, s in enumerate(singles):
        assert np.array_equal(b.get_planes(i), s.get_planes()), i
        assert list(last[:, i]) == s.stats()["jacobi_iters"], i
        s.close()
    assert blk == 4 and tot > int(last.sum()) > 0
    b.close()


def test_batch_autotune_keeps_results(gpu):
    swm = gpu
    ms = members()[:3]
    outs, blocks = [], []
    for block in (0, 2):
        b = swm.Batch([params(swm, c, "split", block) for c in ms])
        for i, c in enumerate(ms):
            b.set_planes(i, cases.cell_averages(c))
        b.step()
        b.step()
        blocks.append(b.stats()[0])
        outs.append([b.get_planes(i) for i in range(len(ms))])
        b.close()
    assert blocks[0] in (2, 4, 8) and blocks[1] == 2
    for a, c in zip(outs[0], outs[1]):
        assert np.array_equal(a, c)


def test_batch_rejects_mixed_precision(gpu):
    swm = gpu
    ms = members()[:2]
    ps = [params(swm, ms[0], "split", 4), params(swm, ms[1], "fp64", 4)]
    with pytest.raises(swm.SwmError) as e:
        swm.Batch(ps)
    assert e.value.code == -1
