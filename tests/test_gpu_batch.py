"""Ensembles (swm_batch_*): every member of a batched step is bit-identical to the
same problem stepped alone with the same precision and solver (the ensemble step
kernel runs the single-grid tile, assembly and Jacobi code per problem, dt per
problem comes from the same formula on the device), FP64 members are bit-identical
to the oracle, the persistent step (one launch) and the one-launch-per-phase step
agree bit for bit, and the autotuner's choice does not change results."""
import numpy as np
import pytest

import cases
import oracle as O

pytestmark = pytest.mark.gpu


def members():
    out = []
    # uneven sizes, odd row pitches among them (rows padded to an even pitch for the
    # Jacobi tiles); 66 and 129 leave edge tiles two and one columns wide, which the
    # ensemble loads and sweeps as partial tiles and the single grid as full ones
    for name, n in (("vortex", 40), ("dambreak", 57), ("lake", 73), ("island", 50),
                    ("lake_dry", 41), ("vortex", 66), ("island", 129)):
        c = cases.case(name, n=n)
        c["well_balanced"] = 0
        out.append(c)
    return out


def params(swm, c, precision, block):
    return swm.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                           bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"],
                           precision=precision, solver="stencil", jacobi_block=block)


@pytest.mark.parametrize("precision", ["fp64", "split", "fp64_fma"])
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


def test_batch_is_one_launch_per_step(gpu):
    swm = gpu
    ms = members()[:2]
    b = swm.Batch([params(swm, c, "split", 4) for c in ms])
    for i, c in enumerate(ms):
        b.set_planes(i, cases.cell_averages(c))
    b.step()
    launches, ctas = b.launch_info()
    assert launches == 1 and ctas >= 148
    b.set_launches(True)
    assert b.launch_info() == (17, 0)
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_persistent_and_per_phase_steps_identical(gpu, precision):
    swm = gpu
    ms = members()
    outs = []
    for per_phase in (False, True):
        b = swm.Batch([params(swm, c, precision, 4) for c in ms])
        b.set_launches(per_phase)
        for i, c in enumerate(ms):
            b.set_planes(i, cases.cell_averages(c))
        dts = [b.step()[0] for _ in range(3)]
        outs.append(([b.get_planes(i) for i in range(len(ms))], dts, b.stats()[2]))
        b.close()
    for a, c in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(a, c)
    assert all(np.array_equal(x, y) for x, y in zip(outs[0][1], outs[1][1]))
    assert np.array_equal(outs[0][2], outs[1][2])


def test_autotuned_step_form_matches_fixed_forms(gpu):
    # jacobi_block = 0: the first step times the persistent and the per-phase forms (and
    # the sweeps per pass), restoring the state after each; whichever it keeps, the
    # steps equal those of a batch with the form and block fixed
    swm = gpu
    ms = members()[:4]
    outs = []
    for block, per_phase in ((0, None), (4, False)):
        b = swm.Batch([params(swm, c, "split", block) for c in ms])
        b.set_launches(per_phase)
        for i, c in enumerate(ms):
            b.set_planes(i, cases.cell_averages(c))
        for _ in range(2):
            b.step()
        if block == 0:
            assert b.launch_info()[0] in (1, 17)
        outs.append([b.get_planes(i) for i in range(len(ms))])
        b.close()
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


def test_phase_times_step_like_a_step_in_both_forms(gpu):
    # the timed step of either form advances the state exactly as step() does
    swm = gpu
    ms = members()[:3]
    outs = []
    for how in ("step", "persistent", "phased"):
        b = swm.Batch([params(swm, c, "split", 4) for c in ms])
        if how != "step":
            b.set_launches(how == "phased")
        for i, c in enumerate(ms):
            b.set_planes(i, cases.cell_averages(c))
        if how == "step":
            b.step()
        else:
            pt = b.phase_times()
            assert len(pt) == 16 and all(v > 0.0 for v in pt.values()), (how, pt)
        outs.append([b.get_planes(i) for i in range(len(ms))])
        b.close()
    for other in outs[1:]:
        for x, y in zip(outs[0], other):
            assert np.array_equal(x, y)


def test_per_phase_launch_counts(gpu):
    swm = gpu
    ms = members()[:2]
    for precision, n in (("split", 17), ("fp64_fma", 17), ("fp64", 25)):
        b = swm.Batch([params(swm, c, precision, 4) for c in ms])
        b.set_launches(True)
        assert b.launch_info() == (n, 0), precision
        b.close()


def test_fp64_members_match_the_oracle(gpu):
    # members of uneven size and family, stepped in one ensemble, against the oracle
    swm = gpu
    # 65 and 130 leave Jacobi edge tiles one and two columns wide
    ms = [cases.case("vortex", n=48, seed=1), cases.case("dambreak", n=70),
          cases.case("island", n=64), cases.case("lake", n=90), cases.case("vortex", n=65),
          cases.case("dambreak", n=130)]
    for c in ms:
        c["well_balanced"] = 0
    b = swm.Batch([params(swm, c, "fp64", 0) for c in ms])
    oracles = []
    for i, c in enumerate(ms):
        P = cases.cell_averages(c)
        b.set_planes(i, P)
        o = O.Oracle(O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"], cfl=c["cfl"],
                                   bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"]))
        o.set_planes(P)
        oracles.append(o)
    for step in range(4):
        dts, rc = b.step()
        assert rc == 0
        for i, o in enumerate(oracles):
            dt = o.timestep()
            assert dt == dts[i], (step, i)
            o.step(0.0, dt)
    for i, o in enumerate(oracles):
        assert np.array_equal(b.get_planes(i), o.get_planes()), i
    b.close()
