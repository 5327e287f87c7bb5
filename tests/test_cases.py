"""Benchmark cases: the numpy initial-condition fill (driver side, used by the
bench) agrees with the oracle's restatement of FillInitialConditions, the
ghosted layout round-trips, and the ensemble generator follows its spec."""
import numpy as np
import pytest

import cases
import oracle as O


@pytest.mark.parametrize("name", ["vortex", "lake", "lake_dry", "dambreak", "island"])
def test_cell_averages_match_oracle(name):
    c = cases.case(name, n=24)
    p = O.make_params(c["nx"], c["ny"], c["x0"], c["x1"], g=c["g"],
                      bathy_flag=c["bathy_flag"], bathy_par=c["bathy_par"])
    o = O.Oracle(p)
    o.fill_ic(c["ic"], c["par"])
    ref = o.get_planes()
    got = cases.cell_averages(c)
    assert np.allclose(got, ref, rtol=1e-15, atol=1e-15)


def test_ghosted_roundtrip_and_periodic_frame():
    rng = np.random.default_rng(0)
    P = rng.random((3, 5, 7))
    G = cases.ghosted(P)
    assert G.shape == (11, 13, 3)
    assert np.array_equal(cases.planes_of(G), P)
    # U(:,-2,jj) = U(:,nx-2,jj) (equation.f90:557-559): ghost column 0 is interior nx-3
    assert np.array_equal(G[3:-3, 0, :], P[:, :, 7 - 3].T)
    assert np.array_equal(G[0, 3:-3, :], P[:, 5 - 3, :].T)


def test_ensemble_spec():
    ens = cases.ensemble(seed=0)
    assert len(ens) == 256
    sides = np.array([c["nx"] for c in ens])
    assert sides.min() >= 64 and sides.max() <= 512
    fams = {c["family"] for c in ens}
    assert fams == {"vortex", "dambreak", "lake"}
    total = sum(c["nx"] * c["ny"] for c in ens)
    assert 5e6 < total < 4e7
    assert cases.ensemble(seed=0)[17]["par"] == ens[17]["par"]


def test_island_dry_patch_and_hump():
    c = cases.case("island", n=64)
    P = cases.cell_averages(c)
    assert P[0].min() == pytest.approx(1e-6, rel=1e-12)  # dry top of the island
    assert P[1].max() > 0.5  # incoming hump carries momentum
