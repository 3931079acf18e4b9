"""Committee of potentials (globalHdnnpEnergyAndForces, globalHdnnps.f90:31-70).

Members share the first member's neighbour lists and scaled symmetry
functions; energy, forces and dE/dh are member means and std the population
standard deviation of the member energies.  Checked through the C ABI:
* against the FP64 oracle run member by member (members with the same
  scaling.data, so each oracle run equals the reference's member evaluation):
  |dE| <= 1e-10 |E|, max |dF|, |d dEdLat| <= 1e-9, |d std| <= 1e-9;
* a member's own scaling.data is ignored (the reference scales with member 1's);
* a committee of one equals the plain evaluation bitwise;
* the mixed-precision committee stays within 1e-6 Ha/atom and 1e-5 Ha/Bohr;
* mismatched members and a context of another potential are rejected.
"""
import os
import shutil

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def member_dirs(tmp_path_factory, W):
    dirs = [ABX3_DIR]
    for seed in (7, 8):
        d = str(tmp_path_factory.mktemp(f"member{seed}"))
        for f in ("input.nn", "scaling.data"):
            shutil.copy(os.path.join(ABX3_DIR, f), d)
        W.write_abx3_weights(d, seed=seed)
        dirs.append(d)
    return dirs


@pytest.fixture(scope="module")
def members(pkg, member_dirs):
    from hdnnp_b200 import engine

    ms = [engine.Hdnnp.from_runner(d) for d in member_dirs]
    yield ms
    for m in ms:
        m.close()


def oracle_committee(orc, dirs, s):
    res = [orc.Model(d).eval(s["Z"], s["pos"], s["lat"]) for d in dirs]
    E = np.array([r["energy"] for r in res])
    F = np.mean([r["forces"] for r in res], axis=0)
    L = np.mean([r["dEdLat"] for r in res], axis=0) if s["lat"] is not None else None
    return E.mean(), F, L, np.sqrt(np.mean((E - E.mean()) ** 2))


def test_committee_vs_oracle(members, member_dirs, orc, W):
    from hdnnp_b200 import engine

    lead = members[0]
    for s in [W.config_c2(), W.config_c4(n_struct=1, seed=31)[0]]:
        E, F, L, sd = lead.committee_energy_and_forces(members, engine.AtStruct(s["Z"], s["pos"], s["lat"]),
                                                       dEdLat=True)
        Er, Fr, Lr, sdr = oracle_committee(orc, member_dirs, s)
        assert abs(E - Er) <= 1e-10 * abs(Er)
        assert np.abs(F - Fr).max() <= 1e-9
        assert np.abs(L - Lr).max() <= 1e-9
        assert abs(sd - sdr) <= 1e-9 and sd > 1e-6  # the members really differ


def test_committee_batch_and_molecule(members, member_dirs, orc, W):
    structs = W.config_c4(n_struct=6, seed=32)
    mol = W.abx3_cell()
    structs.append({"Z": mol["Z"], "pos": mol["pos"], "lat": None})
    out = members[0].committee_eval_batch(members, structs, dEdLat=True)
    off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
    for k, s in enumerate(structs):
        Er, Fr, Lr, sdr = oracle_committee(orc, member_dirs, s)
        assert abs(out["energy"][k] - Er) <= 1e-10 * abs(Er)
        assert np.abs(out["forces"][off[k]:off[k + 1]] - Fr).max() <= 1e-9
        assert abs(out["std"][k] - sdr) <= 1e-9
        if Lr is not None:
            assert np.abs(out["dEdLat"][9 * k:9 * k + 9].reshape(3, 3, order="F") - Lr).max() <= 1e-9
        else:
            assert not np.any(out["dEdLat"][9 * k:9 * k + 9])


def test_member_scaling_is_ignored(pkg, members, member_dirs, tmp_path, W):
    """The reference scales the symmetry functions with member 1's scaling
    for every member; a member's own scaling.data plays no part."""
    from hdnnp_b200 import engine

    d = str(tmp_path / "rescaled")
    shutil.copytree(member_dirs[1], d)
    lines = open(os.path.join(d, "scaling.data")).read().splitlines()
    out = []
    for ln in lines[:-1]:  # last line: energy min/max
        f = ln.split()
        out.append(" ".join(f[:2] + [repr(float(x) * 1.5 + 0.1) for x in f[2:]]))
    open(os.path.join(d, "scaling.data"), "w").write("\n".join(out + lines[-1:]) + "\n")
    other = engine.Hdnnp.from_runner(d)
    s = W.config_c2()
    ats = engine.AtStruct(s["Z"], s["pos"], s["lat"])
    a = members[0].committee_energy_and_forces(members[:2], ats, dEdLat=True)
    b = members[0].committee_energy_and_forces([members[0], other], ats, dEdLat=True)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]
    # while the member alone does see its own scaling
    assert other.energy_and_forces(ats)[0] != members[1].energy_and_forces(ats)[0]
    other.close()


def test_committee_of_one_is_plain(members, W):
    from hdnnp_b200 import engine

    s = W.config_c2()
    ats = engine.AtStruct(s["Z"], s["pos"], s["lat"])
    E, F, L, sd = members[0].committee_energy_and_forces(members[:1], ats, dEdLat=True)
    E0, F0, L0 = members[0].energy_and_forces(ats, dEdLat=True)
    assert E == E0 and np.array_equal(F, F0) and np.array_equal(L, L0) and sd == 0.0


def test_committee_mixed_precision(members, member_dirs, orc, W):
    from hdnnp_b200 import engine

    lead = members[0]
    s = W.config_c2()
    lead.set_precision(engine.HDNNP_PREC_MIXED)
    try:
        E, F, L, sd = lead.committee_energy_and_forces(members, engine.AtStruct(s["Z"], s["pos"], s["lat"]),
                                                       dEdLat=True)
    finally:
        lead.set_precision(engine.HDNNP_PREC_FP64)
    Er, Fr, Lr, sdr = oracle_committee(orc, member_dirs, s)
    n = len(s["Z"])
    print(f"mixed committee: |dE|/atom {abs(E - Er) / n:.2e}  max|dF| {np.abs(F - Fr).max():.2e}")
    assert abs(E - Er) / n <= 1e-6 and np.abs(F - Fr).max() <= 1e-5
    assert np.abs(L - Lr).max() / n <= 1e-5 and abs(sd - sdr) / n <= 1e-6


def test_committee_errors(pkg, members, W):
    from hdnnp_b200 import engine
    from hdnnp_b200.engine import HdnnpError

    ex = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    s = W.config_c2()
    ats = engine.AtStruct(s["Z"], s["pos"], s["lat"])
    with pytest.raises(HdnnpError) as e:  # other elements
        members[0].committee_energy_and_forces([members[0], ex], ats)
    assert e.value.code == 1
    with pytest.raises(HdnnpError) as e:  # context of another potential than members[0]
        members[1].committee_energy_and_forces(members, ats)
    assert e.value.code == 1
    ex.close()
    # the context still works after the rejected calls
    E, F, L, sd = members[0].committee_energy_and_forces(members, ats)
    assert np.isfinite(E) and sd > 0
