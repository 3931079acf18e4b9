"""Pins the FP64 oracle (oracle/hdnnp_oracle.cpp).

The reference ships no golden outputs and cannot be compiled here (no Fortran
compiler), so the oracle is checked against: an independent torch-autograd
restatement (tests/indep_torch.py), central finite differences, the
reference's own internal cross-check routines (single-SF vs fused SFs,
O(N^2) vs cell-list neighbours), invariances, and the committed fixtures.
"""
import json
import os

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR, GOLDEN


def small_cell(W, seed=7, strain=0.05, jitter=0.15):
    rng = np.random.default_rng(seed)
    c = W.strain(W.abx3_cell(), rng.uniform(-strain, strain, (3, 3)))
    c["pos"] = c["pos"] + rng.normal(0, jitter, c["pos"].shape)
    return c


def test_parse_example(ex_model):
    assert ex_model.elements == [1, 6, 7]
    assert ex_model.nsf == {1: 31, 6: 18, 7: 18}
    assert ex_model.max_rc == 12.0
    s, c, _ = ex_model.flags()
    assert s and c
    sf = ex_model.sfs(1)
    # radial SFs first, sorted by the formatted key (eta, then element)
    assert (sf[:15, 0] == 2).all() and (sf[15:, 0] == 3).all()
    assert list(sf[:3, 1]) == [1, 6, 7] and sf[0, 4] == 0.004
    net = ex_model.net(6)
    assert [W.shape for W, _, _ in net] == [(10, 18), (10, 10), (1, 10)]
    assert "".join(a for _, _, a in net) == "ttl"


def test_parser_errors(orc, tmp_path):
    src = open(os.path.join(EXAMPLE_DIR, "input.nn")).read()
    bad = src.replace("number_of_elements 3\nelements N C H", "elements N C H\nnumber_of_elements 3")
    d = tmp_path / "p1"
    d.mkdir()
    (d / "input.nn").write_text(bad)
    with pytest.raises(orc.OracleError, match="number_of_elements"):
        orc.Model(str(d))
    with pytest.raises(orc.OracleError, match="not found"):
        orc.Model(str(tmp_path / "missing"))
    # reference cap of 200 SFs per element (hdnnps.f90:48)
    with pytest.raises(orc.OracleError, match="nmaxSFs"):
        orc.Model(ABX3_DIR, cap_sfs=200)
    # scaling index mismatch (hdnnps.f90:289-292)
    d2 = tmp_path / "p2"
    d2.mkdir()
    for f in os.listdir(EXAMPLE_DIR):
        (d2 / f).write_bytes(open(os.path.join(EXAMPLE_DIR, f), "rb").read())
    sc = (d2 / "scaling.data").read_text().splitlines()
    sc[0] = sc[0].replace("   1    1", "   1    2", 1)
    (d2 / "scaling.data").write_text("\n".join(sc) + "\n")
    with pytest.raises(orc.OracleError, match="wrong index"):
        orc.Model(str(d2))


def test_fd_forces_example(ex_model, c1):
    s, _, _ = c1
    r = ex_model.eval(s["Z"], s["pos"])
    h = 1e-5
    fd = np.zeros_like(s["pos"])
    for i in range(len(s["Z"])):
        for d in range(3):
            p = s["pos"].copy()
            p[i, d] += h
            ep = ex_model.eval(s["Z"], p)["energy"]
            p[i, d] -= 2 * h
            em = ex_model.eval(s["Z"], p)["energy"]
            fd[i, d] = -(ep - em) / (2 * h)
    assert np.abs(fd - r["forces"]).max() < 1e-8


def test_fd_forces_and_dEdLat_small_cell(abx3_model, W):
    c = small_cell(W)
    r = abx3_model.eval(c["Z"], c["pos"], c["lat"])
    h = 1e-5
    fd = np.zeros_like(c["pos"])
    for i in range(len(c["Z"])):
        for d in range(3):
            p = c["pos"].copy()
            p[i, d] += h
            ep = abx3_model.eval(c["Z"], p, c["lat"])["energy"]
            p[i, d] -= 2 * h
            em = abx3_model.eval(c["Z"], p, c["lat"])["energy"]
            fd[i, d] = -(ep - em) / (2 * h)
    assert np.abs(fd - r["forces"]).max() < 1e-8 * max(1.0, np.abs(r["forces"]).max())
    frac = np.linalg.solve(c["lat"], c["pos"].T).T
    fdl = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            L = c["lat"].copy()
            L[a, b] += h
            ep = abx3_model.eval(c["Z"], frac @ L.T, L)["energy"]
            L[a, b] -= 2 * h
            em = abx3_model.eval(c["Z"], frac @ L.T, L)["energy"]
            fdl[a, b] = (ep - em) / (2 * h)
    assert np.abs(fdl - r["dEdLat"]).max() < 1e-8 * max(1.0, np.abs(r["dEdLat"]).max())


@pytest.mark.parametrize("case", ["example", "small_cell", "prz_cell"])
def test_independent_autograd(case, ex_model, abx3_model, prz_model, c1, W):
    """prz_cell: softplus/ReLU layers and non-integer zeta (the real-power
    branch, symmetryFunctions.f90:266-273; activations
    neuralNetworks.f90:45-49,69-80)."""
    import indep_torch as T

    if case == "example":
        m, s = ex_model, c1[0]
    elif case == "small_cell":
        m, s = abx3_model, small_cell(W, seed=11)
    else:
        m, s = prz_model, small_cell(W, seed=12)
    desc = T.describe(m)
    E, F, dl = T.energy_forces_dEdLat(desc, s["Z"], s["pos"], s["lat"])
    r = m.eval(s["Z"], s["pos"], s["lat"])
    assert abs(E - r["energy"]) <= 1e-11 * abs(r["energy"])
    assert np.abs(F - r["forces"]).max() <= 1e-10 * max(1.0, np.abs(F).max())
    if dl is not None:
        assert np.abs(dl - r["dEdLat"]).max() <= 1e-10 * max(1.0, np.abs(dl).max())


def _nei_set(counts, idx, npos):
    out = []
    for i in range(len(counts)):
        s = sorted((int(idx[i, q]), tuple(np.round(npos[i, q], 6))) for q in range(counts[i]))
        out.append(s)
    return out


@pytest.mark.parametrize("case", ["molecule", "small_cell", "c2"])
def test_grid_vs_brute_neighbours(case, ex_model, abx3_model, c1, W):
    if case == "molecule":
        m, s = ex_model, c1[0]
    elif case == "small_cell":
        m, s = abx3_model, small_cell(W)
    else:
        m, s = abx3_model, W.config_c2()
    a = m.neighbours(s["Z"], s["pos"], s["lat"])
    b = m.neighbours(s["Z"], s["pos"], s["lat"], brute=True)
    assert (a[0] == b[0]).all()
    assert _nei_set(*a) == _nei_set(*b)
    # entry 0 is the atom itself
    assert (a[1][:, 0] == np.arange(len(s["Z"]))).all()


@pytest.mark.parametrize("case", ["example", "small_cell", "prz_cell"])
def test_fused_vs_single_sf(case, ex_model, abx3_model, prz_model, c1, W):
    m, s = {"example": (ex_model, c1[0]), "small_cell": (abx3_model, small_cell(W)),
            "prz_cell": (prz_model, small_cell(W, seed=13))}[case]
    cap = int(m.neighbours(s["Z"], s["pos"], s["lat"])[0].max())
    G1, d1 = m.symfunctions(s["Z"], s["pos"], s["lat"], with_grad=True, cap=cap)
    G2, d2 = m.symfunctions(s["Z"], s["pos"], s["lat"], separate=True, with_grad=True, cap=cap)
    assert np.abs(G1 - G2).max() < 1e-12 * max(1, np.abs(G1).max())
    assert np.abs(d1 - d2).max() < 1e-12 * max(1, np.abs(d1).max())


def test_invariances(ex_model, abx3_model, c1, W):
    s = c1[0]
    r0 = ex_model.eval(s["Z"], s["pos"])
    # translation + rotation of a molecule
    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    p = s["pos"] @ q.T + np.array([1.3, -2.0, 0.7])
    r1 = ex_model.eval(s["Z"], p)
    assert abs(r1["energy"] - r0["energy"]) < 1e-12 * abs(r0["energy"])
    assert np.abs(r1["forces"] - r0["forces"] @ q.T).max() < 1e-11
    # permutation
    perm = rng.permutation(len(s["Z"]))
    r2 = ex_model.eval(s["Z"][perm], s["pos"][perm])
    assert abs(r2["energy"] - r0["energy"]) < 1e-12 * abs(r0["energy"])
    assert np.abs(r2["forces"] - r0["forces"][perm]).max() < 1e-12
    # supercell extensivity: E(2x2x2) = 8 E(cell), forces repeat
    c = small_cell(W, seed=5)
    rc = abx3_model.eval(c["Z"], c["pos"], c["lat"])
    big = W.supercell(c, (2, 2, 2))
    rb = abx3_model.eval(big["Z"], big["pos"], big["lat"])
    assert abs(rb["energy"] - 8 * rc["energy"]) < 1e-11 * abs(rb["energy"])
    assert np.abs(rb["forces"] - np.tile(rc["forces"], (8, 1))).max() < 1e-10
    # dEdLat of the supercell: h_big = 2 h  ->  dE/dh_big = 8 * dE/dh / 2
    assert np.abs(rb["dEdLat"] - 4 * rc["dEdLat"]).max() < 1e-9 * np.abs(rb["dEdLat"]).max()


def test_golden_fixtures(ex_model, abx3_model, c1, W):
    with open(os.path.join(GOLDEN, "oracle_fixtures.json")) as f:
        fx = json.load(f)
    s = c1[0]
    r = ex_model.eval(s["Z"], s["pos"])
    assert abs(r["energy"] - fx["c1"]["energy"]) < 1e-12 * abs(fx["c1"]["energy"])
    assert np.abs(r["forces"] - np.array(fx["c1"]["forces"])).max() < 1e-12
    c = small_cell(W)
    r = abx3_model.eval(c["Z"], c["pos"], c["lat"])
    assert abs(r["energy"] - fx["cell"]["energy"]) < 1e-12 * abs(fx["cell"]["energy"])
    assert np.abs(r["forces"] - np.array(fx["cell"]["forces"])).max() < 1e-11
    assert np.abs(r["dEdLat"] - np.array(fx["cell"]["dEdLat"])).max() < 1e-11


def test_reference_double_wrap_of_face_atoms(abx3_model, W):
    """A quirk of the reference the oracle keeps: hdnnpCalcNeighborLists wraps
    a periodic structure (hdnnps.f90:379-386) and buildNeighborListGrid wraps
    that copy again (neighborLists.f90:157), but takes each centre's own
    position from the first copy (:125) and its neighbours from the second.
    For an atom whose fractional coordinate rounds to 1.0 in the first wrap
    the second wrap moves it by a lattice vector, so its environment is seen
    with inconsistent images.  The unjittered strained ABX3 lattice has such
    atoms (fractional 0 to rounding): there the grid path's energy per atom
    depends on the supercell size, while a rigidly translated copy (no atom on
    a face) and the brute-force list (neighborLists.f90:21-81, one wrap) agree
    with each other for every size.  The engine wraps once, as the translated
    copy."""
    shift = np.array([0.0137, 0.0213, 0.0071])
    per_atom = []
    for n in (2, 3):
        s = W.config_c3(n=n)
        nat = len(s["Z"])
        grid = abx3_model.eval(s["Z"], s["pos"], s["lat"])["energy"] / nat
        moved = abx3_model.eval(s["Z"], s["pos"] + shift, s["lat"])["energy"] / nat
        brute = abx3_model.eval(s["Z"], s["pos"], s["lat"], brute=True)["energy"] / nat
        assert abs(moved - brute) <= 1e-12 * abs(brute)
        per_atom.append((grid, moved))
    assert abs(per_atom[0][1] - per_atom[1][1]) <= 1e-12 * abs(per_atom[0][1])  # translated: size-independent
    assert abs(per_atom[0][0] - per_atom[0][1]) > 1e-4 * abs(per_atom[0][1])  # the quirk shows on the lattice
