"""Structure readers and writers (structio.py) against the reference's file
semantics (src/atoms/atomicStructure.f90), on CPU.

Checked: the reference's own example input.xyz; full-precision round trips of
every format (bitwise for xyz and data, to rounding where Angstrom or
fractional coordinates are involved); the unit conversions (Angstrom in
FHI-aims, POSCAR and 'angstroem' ascii, ang2bohr of constants.f90:7); the
lattice alignment of the ascii writer (distances and fractional coordinates
kept); POSCAR without Direct coordinates and a fourth lattice vector are
rejected; a batch read from files evaluates like the structures it holds
(oracle).
"""
import os

import numpy as np
import pytest

from conftest import EXAMPLE_DIR


@pytest.fixture(scope="module")
def SIO(pkg):
    from hdnnp_b200 import structio

    return structio


def frac(s):
    return np.linalg.solve(s["lat"], s["pos"].T).T


def test_example_xyz(SIO, W):
    a = SIO.read_xyz(os.path.join(EXAMPLE_DIR, "input.xyz"))
    b = W.read_xyz(os.path.join(EXAMPLE_DIR, "input.xyz"))
    assert np.array_equal(a["Z"], b["Z"]) and np.array_equal(a["pos"], b["pos"]) and a["lat"] is None
    assert list(a["Z"]) == [7, 6, 1, 1, 1, 1, 1, 1]
    assert a["pos"][0, 0] == 1.39424 and a["pos"][1, 0] == -1.39424  # read as written, no unit conversion


def test_xyz_and_data_round_trip_bitwise(SIO, W, tmp_path):
    s = W.config_c4(n_struct=3, seed=9)
    SIO.write_xyz(tmp_path / "a.xyz", s[0])
    r = SIO.read_xyz(tmp_path / "a.xyz")
    assert np.array_equal(r["pos"], s[0]["pos"]) and np.array_equal(r["Z"], s[0]["Z"])
    mol = W.abx3_cell()
    structs = s + [{"Z": mol["Z"], "pos": mol["pos"], "lat": None}]
    rng = np.random.default_rng(1)
    E = rng.normal(size=len(structs))
    F = [rng.normal(size=(len(t["Z"]), 3)) for t in structs]
    Q = [rng.normal(size=len(t["Z"])) for t in structs]
    SIO.write_data(tmp_path / "input.data", structs, energies=E, forces=F, charges=Q)
    back = SIO.read_data(tmp_path / "input.data")
    assert len(back) == len(structs)
    for t, u, e, f, q in zip(structs, back, E, F, Q):
        assert np.array_equal(t["pos"], u["pos"]) and np.array_equal(t["Z"], u["Z"])
        assert (t["lat"] is None) == (u["lat"] is None)
        if t["lat"] is not None:
            assert np.array_equal(t["lat"], u["lat"])
        assert u["energy"] == e and np.array_equal(u["forces"], f) and np.array_equal(u["q"], q)
        assert u["charge"] == round(float(np.sum(q)))


def test_angstrom_formats(SIO, W, tmp_path):
    s = W.config_c4(n_struct=1, seed=10)[0]
    for name, wr, rd in (("geometry.in", SIO.write_fhiaims, SIO.read_fhiaims),
                         ("POSCAR", SIO.write_poscar, SIO.read_poscar)):
        wr(tmp_path / name, s)
        r = rd(tmp_path / name)
        assert np.abs(r["lat"] - s["lat"]).max() < 1e-12
        if name == "POSCAR":  # grouped by element: compare as sets of (Z, frac)
            key = lambda t: sorted(zip(t["Z"].tolist(), np.round(frac(t) % 1.0, 9).tolist()))
            assert key(r) == key(s)
        else:
            assert np.array_equal(r["Z"], s["Z"]) and np.abs(r["pos"] - s["pos"]).max() < 1e-12
    # units: one Angstrom in the file is ang2bohr Bohr
    (tmp_path / "g.in").write_text("lattice_vector 2 0 0\nlattice_vector 0 2 0\nlattice_vector 0 0 2\natom 1 0 0 H\n")
    g = SIO.read_fhiaims(tmp_path / "g.in")
    assert g["pos"][0, 0] == 1.8897259886 and g["lat"][0, 0] == 2 * 1.8897259886


def test_ascii_alignment(SIO, W, tmp_path):
    s = W.strain(W.supercell(W.abx3_cell(), (1, 2, 1)), np.array([[0.02, 0.03, -0.01], [0.0, -0.02, 0.04],
                                                                   [0.05, 0.01, 0.0]]))
    for angs in (False, True):
        SIO.write_ascii(tmp_path / "a.ascii", s, to_angstrom=angs)
        r = SIO.read_ascii(tmp_path / "a.ascii")
        L = r["lat"]
        assert L[1, 0] == 0 and L[2, 0] == 0 and L[2, 1] == 0  # vector 1 along x, vector 2 in the xy plane
        assert np.abs(L.T @ L - s["lat"].T @ s["lat"]).max() < 1e-10  # same cell up to a rotation
        assert np.abs(frac(r) - frac(s)).max() < 1e-12
        d0 = np.linalg.norm(s["pos"][:, None] - s["pos"][None], axis=-1)
        d1 = np.linalg.norm(r["pos"][:, None] - r["pos"][None], axis=-1)
        assert np.abs(d0 - d1).max() < 1e-10


def test_rejects(SIO, tmp_path):
    (tmp_path / "POSCAR").write_text("c\n1.0\n1 0 0\n0 1 0\n0 0 1\nH\n1\nCartesian\n0 0 0\n")
    with pytest.raises(ValueError):
        SIO.read_poscar(tmp_path / "POSCAR")
    (tmp_path / "g.in").write_text("".join("lattice_vector 1 0 0\n" for _ in range(4)))
    with pytest.raises(ValueError):
        SIO.read_fhiaims(tmp_path / "g.in")
    assert SIO.sym_to_z("Xx") == -1 and SIO.z_to_sym(119) == "XX"


def test_batch_from_files_matches_oracle(SIO, W, abx3_model, tmp_path):
    s = W.config_c4(n_struct=2, seed=12)
    SIO.write_data(tmp_path / "a.data", s)
    SIO.write_poscar(tmp_path / "POSCAR", s[0])
    batch = SIO.read_batch([tmp_path / "a.data"], "data") + SIO.read_batch([tmp_path / "POSCAR"], "poscar")
    for t, u in zip(batch, [s[0], s[1], s[0]]):
        ea = abx3_model.eval(t["Z"], t["pos"], t["lat"])["energy"]
        eb = abx3_model.eval(u["Z"], u["pos"], u["lat"])["energy"]
        assert abs(ea - eb) <= 1e-10 * abs(eb)
