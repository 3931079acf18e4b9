"""The stage-level entry points, chained as the reference's own callers chain
them (hdnnpEnergyAndForces, hdnnps.f90:346-368; globalHdnnpEnergyAndForces,
globalHdnnps.f90:47-57), through the C ABI:

* hdnnp_calc_neighbor_lists -> hdnnp_calc_symfunctions -> hdnnp_calc_nns
  gives bitwise the energy, forces and dE/dh of hdnnp_energy_and_forces (FP64
  and mixed), and the values G bitwise those of the fused call;
* one set of lists and values with every committee member's networks
  (hdnnp_calc_nns with another potential) averages to the committee entry
  point's result (to rounding: that one averages dE/dG before one
  contraction) and each member equals the FP64 oracle;
* calls out of order return HDNNP_E_STATE;
* the type(hdnnp) components (hdnnps.f90:13-21) read back as the oracle
  parsed them.
"""
import os
import shutil

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng(pkg):
    from hdnnp_b200 import engine

    return engine


def cases(W, c1):
    rng = np.random.default_rng(71)
    cell = W.strain(W.supercell(W.abx3_cell(), (2, 1, 1)), rng.uniform(-0.04, 0.04, (3, 3)))
    cell["pos"] = cell["pos"] + rng.normal(0, 0.1, cell["pos"].shape)
    return [(EXAMPLE_DIR, c1[0]), (ABX3_DIR, cell), (ABX3_DIR, W.config_c2(seed=72))]


@pytest.mark.parametrize("precision", [0, 1])
def test_chained_stages_equal_the_fused_call(eng, W, c1, precision):
    for d, s in cases(W, c1):
        pot = eng.Hdnnp.from_runner(d)
        try:
            pot.set_precision(precision)
            pot.set_option("small_eval", 0)  # molecules through the general pipeline, like the stages
            per = s["lat"] is not None
            ats = eng.AtStruct(s["Z"], s["pos"], s["lat"])
            E0, F0, L0 = pot.energy_and_forces(ats, dEdLat=per)
            nsf = max(pot.nsf.values())
            G0 = pot.fetch("G", len(s["Z"]) * nsf).reshape(-1, nsf) if precision == 0 else None
            ne = pot.calc_neighbor_lists(ats)
            assert ne == int(pot.fetch("nei_count", len(s["Z"]), np.int32).sum())
            G = pot.calc_symfunctions()
            if G0 is not None:
                assert np.array_equal(G, G0)
            E1, F1, L1 = pot.calc_nns(dEdLat=per)
            assert E1 == E0 and np.array_equal(F1, F0), (d, precision)
            if per:
                assert np.array_equal(L1, L0)
            # the networks again on the same values (the committee's loop)
            E2, F2, _ = pot.calc_nns()
            assert E2 == E0 and np.array_equal(F2, F0)
        finally:
            pot.close()


def test_committee_through_stages(eng, W, orc, tmp_path):
    dirs = [ABX3_DIR]
    for seed in (7, 8):
        d = tmp_path / f"m{seed}"
        d.mkdir()
        for f in ("input.nn", "scaling.data"):
            shutil.copy(os.path.join(ABX3_DIR, f), d)
        W.write_abx3_weights(str(d), seed=seed)
        dirs.append(str(d))
    pots = [eng.Hdnnp.from_runner(d) for d in dirs]
    s = W.config_c2(seed=73)
    ats = eng.AtStruct(s["Z"], s["pos"], s["lat"])
    try:
        head = pots[0]
        head.calc_neighbor_lists(ats)
        head.calc_symfunctions(fetch=False)
        res = [head.calc_nns(nn=p, dEdLat=True) for p in pots]
        for (E, F, L), d in zip(res, dirs):
            ref = orc.Model(d).eval(s["Z"], s["pos"], s["lat"])
            assert abs(E - ref["energy"]) <= 1e-10 * abs(ref["energy"])
            assert np.abs(F - ref["forces"]).max() <= 1e-9
            assert np.abs(L - ref["dEdLat"]).max() <= 1e-9
        Ec, Fc, Lc, sd = head.committee_energy_and_forces(pots, ats, dEdLat=True)
        Em = np.mean([r[0] for r in res])
        assert abs(Ec - Em) <= 1e-10 * abs(Em)
        assert np.abs(Fc - np.mean([r[1] for r in res], axis=0)).max() <= 1e-9
        assert np.abs(Lc - np.mean([r[2] for r in res], axis=0)).max() <= 1e-9
        assert abs(sd - np.std([r[0] for r in res])) <= 1e-9
    finally:
        for p in pots:
            p.close()


def test_stage_order_errors(eng, W):
    pot = eng.Hdnnp.from_runner(ABX3_DIR)
    ex = eng.Hdnnp.from_runner(EXAMPLE_DIR)
    s = W.config_c2(seed=74)
    ats = eng.AtStruct(s["Z"], s["pos"], s["lat"])
    try:
        with pytest.raises(eng.HdnnpError) as e:
            pot._stage_nat = len(s["Z"])
            pot.calc_symfunctions()
        assert e.value.code == 6
        pot.calc_neighbor_lists(ats)
        with pytest.raises(eng.HdnnpError) as e:
            pot.calc_nns()
        assert e.value.code == 6
        pot.calc_symfunctions(fetch=False)
        with pytest.raises(eng.HdnnpError) as e:
            pot.calc_nns(nn=ex)  # other elements
        assert e.value.code == 1
        pot.calc_nns()
        pot.energy_and_forces(ats)  # a full evaluation replaces the stage lists
        with pytest.raises(eng.HdnnpError) as e:
            pot.calc_nns()
        assert e.value.code == 6
        mol = eng.AtStruct(s["Z"][:12], s["pos"][:12])
        pot.calc_neighbor_lists(mol)
        pot.calc_symfunctions(fetch=False)
        with pytest.raises(eng.HdnnpError) as e:
            pot.calc_nns(dEdLat=True)  # dE/dh of a molecule
        assert e.value.code == 1
    finally:
        pot.close()
        ex.close()


def test_model_components_read_back(eng, orc):
    for d in (EXAMPLE_DIR, ABX3_DIR):
        pot = eng.Hdnnp.from_runner(d)
        m = orc.Model(d)
        try:
            f = pot.flags()
            sc, ce, ae = m.flags()
            assert f["scalesf"] == sc and f["centersf"] == ce
            assert np.array_equal(f["atomenergies"], ae[1:119])
            for z in m.elements:
                assert np.array_equal(pot.symfunctions(z), m.sfs(z))
                for (W1, b1, a1), (W2, b2, a2) in zip(pot.network(z), m.net(z)):
                    assert a1 == a2 and np.array_equal(W1, W2) and np.array_equal(b1, b2)
        finally:
            pot.close()


def test_neighbor_lists_in_reference_layout(eng, W, orc, c1):
    """hdnnp_neighbor_lists_fetch returns the reference's neighborList:
    entry 1 the atom itself, then its neighbours with their Cartesian image
    positions, in the reference's order (the oracle's buildNeighborListGrid)."""
    for d, s in cases(W, c1)[:2]:
        pot = eng.Hdnnp.from_runner(d)
        m = orc.Model(d)
        try:
            pot.calc_neighbor_lists(eng.AtStruct(s["Z"], s["pos"], s["lat"]))
            lists = pot.neighbor_lists()
            counts, idx, npos = m.neighbours(s["Z"], s["pos"], s["lat"])
            for i, (ii, pp) in enumerate(lists):
                assert len(ii) == counts[i]
                assert np.array_equal(ii, idx[i, :counts[i]])
                assert np.abs(pp - npos[i, :counts[i]]).max() <= 1e-12
        finally:
            pot.close()
