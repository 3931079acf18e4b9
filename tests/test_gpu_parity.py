"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Tolerances of the plain FP64 form: |dE| <= 1e-10 |E|, max |dF| <= 1e-9
Ha/Bohr, max |d dEdLat| <= 1e-9 (and the same for the stress).
"""
import json
import os

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR, GOLDEN

pytestmark = pytest.mark.gpu

E_REL, F_ABS, L_ABS = 1e-10, 1e-9, 1e-9


@pytest.fixture(scope="module")
def eng(pkg):
    from hdnnp_b200 import engine

    return engine


@pytest.fixture(scope="module")
def gex(eng):
    p = eng.Hdnnp.from_runner(EXAMPLE_DIR)
    yield p
    p.close()


@pytest.fixture(scope="module")
def gab(eng):
    p = eng.Hdnnp.from_runner(ABX3_DIR)
    yield p
    p.close()


def small_cell(W, seed=7, strain=0.05, jitter=0.15):
    rng = np.random.default_rng(seed)
    c = W.strain(W.abx3_cell(), rng.uniform(-strain, strain, (3, 3)))
    c["pos"] = c["pos"] + rng.normal(0, jitter, c["pos"].shape)
    return c


def check(E, F, dl, ref):
    assert abs(E - ref["energy"]) <= E_REL * abs(ref["energy"]), (E, ref["energy"])
    assert np.abs(F - ref["forces"]).max() <= F_ABS, np.abs(F - ref["forces"]).max()
    if dl is not None:
        assert np.abs(dl - ref["dEdLat"]).max() <= L_ABS, np.abs(dl - ref["dEdLat"]).max()


def test_example_molecule(eng, gex, ex_model, c1):
    s = c1[0]
    E, F, _ = gex.energy_and_forces(eng.AtStruct(s["Z"], s["pos"]))
    check(E, F, None, ex_model.eval(s["Z"], s["pos"]))
    fx = json.load(open(os.path.join(GOLDEN, "oracle_fixtures.json")))["c1"]
    assert abs(E - fx["energy"]) <= E_REL * abs(fx["energy"])
    assert np.abs(F - np.array(fx["forces"])).max() <= F_ABS


def test_flat_and_linear_molecules(eng, gex, ex_model, c1, pkg):
    """A planar molecule (z extent 0) and a 2-atom one (extent 0 in two
    directions): the artificial box is 2e-4 Bohr thick there, so the cell
    search would span ~10^5 cells; the engine stops at the grid (same list)."""
    from hdnnp_b200 import plan as PL

    s = c1[0]
    flat = s["pos"].copy()
    flat[:, 2] = 0.25
    two = np.array([[0.0, 0.0, 0.0], [2.7, 0.0, 0.0]])
    # the oracle searches every cell like the reference, which for the
    # linear molecule means ~10^10 empty cells: it gets a rotated copy
    R, _ = np.linalg.qr(np.random.default_rng(5).normal(size=(3, 3)))
    gex.set_option("small_eval", 0)  # the general pipeline, compared bitwise with the plan below
    for Z, pos, rot in ((s["Z"], flat, np.eye(3)), (s["Z"][:2], two, R)):
        E, F, _ = gex.energy_and_forces(eng.AtStruct(Z, pos))
        ref = ex_model.eval(Z, pos @ rot.T)
        check(E, F, None, {"energy": ref["energy"], "forces": ref["forces"] @ rot})
        with PL.Plan(gex, [{"Z": Z, "pos": pos, "lat": None}]) as p:  # device-built box
            Ep, Fp, _ = p.results()
        assert Ep[0] == E and np.array_equal(Fp, F)
    gex.set_option("small_eval", 1)


def test_crowded_cell_of_a_sparse_molecule(eng, gab, abx3_model):
    """Two clusters 1000 Bohr apart: the molecule's box is so sparse that its
    grid is coarsened to ~60-Bohr cells, and the 280-atom cluster (4 Bohr
    spacing) lands in one cell -- above the 256 atoms the shared-memory cell
    sort takes, so the in-place fallback orders it."""
    rng = np.random.default_rng(23)
    g = np.stack(np.meshgrid(*[np.arange(7)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = np.concatenate([g[:280] * 4.0 + rng.normal(0.0, 0.1, (280, 3)),
                          1000.0 + g[:20] * 4.0 + rng.normal(0.0, 0.1, (20, 3))])
    Z = rng.choice([1, 6, 7, 53, 82], 300).astype(np.int32)
    E, F, _ = gab.energy_and_forces(eng.AtStruct(Z, pos))
    check(E, F, None, abx3_model.eval(Z, pos))


def test_small_cell_images_and_stress(eng, gab, abx3_model, W, orc):
    c = small_cell(W)
    E, F, dl = gab.energy_and_forces(eng.AtStruct(c["Z"], c["pos"], c["lat"]), dEdLat=True)
    ref = abx3_model.eval(c["Z"], c["pos"], c["lat"])
    check(E, F, dl, ref)
    st = eng.dEdLat_to_stress(c["lat"], dl)
    assert np.abs(st - orc.dEdLat_to_stress(c["lat"], ref["dEdLat"])).max() <= L_ABS
    fx = json.load(open(os.path.join(GOLDEN, "oracle_fixtures.json")))["cell"]
    assert abs(E - fx["energy"]) <= E_REL * abs(fx["energy"])


def test_768_atoms(eng, gab, abx3_model, W):
    s = W.config_c2()
    E, F, dl = gab.energy_and_forces(eng.AtStruct(s["Z"], s["pos"], s["lat"]), dEdLat=True)
    check(E, F, dl, abx3_model.eval(s["Z"], s["pos"], s["lat"]))


def test_stage_outputs(eng, gab, abx3_model, W):
    s = small_cell(W, seed=3)
    gab.energy_and_forces(eng.AtStruct(s["Z"], s["pos"], s["lat"]), dEdLat=True)
    n = len(s["Z"])
    nsf = int(gab.fetch("nsf_max", 1, np.int32)[0])
    G = gab.fetch("G", n * nsf).reshape(n, nsf)
    Gref = abx3_model.symfunctions(s["Z"], s["pos"], s["lat"])
    assert np.abs(G - Gref[:, :nsf]).max() <= 1e-11
    ref = abx3_model.eval(s["Z"], s["pos"], s["lat"], per_atom=True)
    dEdG = gab.fetch("dEdG", n * nsf).reshape(n, nsf)
    assert np.abs(dEdG - ref["dEdG"][:, :nsf]).max() <= 1e-10
    atE = gab.fetch("atom_energy", n)
    assert np.abs(atE - ref["atom_energies"]).max() <= 1e-11
    # neighbour sets (the oracle list includes the atom itself as entry 0)
    cnt = gab.fetch("nei_count", n, np.int32)
    oc, oidx, _ = abx3_model.neighbours(s["Z"], s["pos"], s["lat"])
    assert (cnt == oc - 1).all()
    nidx = gab.fetch("nei_index", int(cnt.sum()), np.int32)
    off = np.concatenate([[0], np.cumsum(cnt)])
    for i in range(n):
        assert list(nidx[off[i]:off[i + 1]]) == list(oidx[i, 1:oc[i]])  # same order as the reference


def test_batch_alone_equals_in_mix(eng, gab, W):
    structs = W.config_c4(n_struct=24, seed=11)
    mix = gab.eval_batch(structs, dEdLat=True)
    off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
    for k in (0, 5, 17, 23):
        alone = gab.eval_batch([structs[k]], dEdLat=True)
        assert alone["energy"][0] == mix["energy"][k]
        assert np.array_equal(alone["forces"], mix["forces"][off[k]:off[k + 1]])
        assert np.array_equal(alone["dEdLat"], mix["dEdLat"][9 * k:9 * k + 9])


def test_mixed_batch_vs_oracle(eng, gab, abx3_model, W):
    structs = W.config_c4(n_struct=16, seed=12)
    structs.append(W.read_xyz(os.path.join(EXAMPLE_DIR, "input.xyz")))  # a molecule in the batch
    structs[-1]["Z"] = np.array([7, 6, 1, 1, 1, 1, 1, 1], np.int32)
    out = gab.eval_batch(structs, dEdLat=True)
    off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
    for k, s in enumerate(structs):
        ref = abx3_model.eval(s["Z"], s["pos"], s["lat"])
        dl = out["dEdLat"][9 * k:9 * k + 9].reshape(3, 3, order="F") if s["lat"] is not None else None
        check(out["energy"][k], out["forces"][off[k]:off[k + 1]], dl, ref)


def test_errors_are_status_codes(eng, gab, W):
    c = small_cell(W)
    bad = dict(c)
    with pytest.raises(eng.HdnnpError, match="not in the potential"):
        Z = c["Z"].copy()
        Z[0] = 8
        gab.energy_and_forces(eng.AtStruct(Z, c["pos"], c["lat"]))
    with pytest.raises(eng.HdnnpError, match="singular"):
        gab.energy_and_forces(eng.AtStruct(c["Z"], c["pos"], np.zeros((3, 3)) + 1.0))
    with pytest.raises(eng.HdnnpError, match="periodic"):
        gab.energy_and_forces(eng.AtStruct(c["Z"], c["pos"]), dEdLat=True)
    with pytest.raises(eng.HdnnpError, match="non-finite"):
        p = c["pos"].copy()
        p[2, 1] = np.nan
        gab.energy_and_forces(eng.AtStruct(c["Z"], p, c["lat"]))
    # the context stays usable after errors
    E, F, _ = gab.energy_and_forces(eng.AtStruct(c["Z"], c["pos"], c["lat"]))
    assert np.isfinite(E)


def test_generic_and_fast_kernels_agree(eng, gab, abx3_model, W):
    s = W.config_c4(n_struct=6, seed=13)
    fast = gab.eval_batch(s, dEdLat=True)
    gab.set_option("generic_sf", 1)
    try:
        gen = gab.eval_batch(s, dEdLat=True)
    finally:
        gab.set_option("generic_sf", 0)
    assert np.abs(fast["energy"] - gen["energy"]).max() <= E_REL * np.abs(gen["energy"]).max()
    assert np.abs(fast["forces"] - gen["forces"]).max() <= F_ABS
    assert np.abs(fast["dEdLat"] - gen["dEdLat"]).max() <= L_ABS


def test_neighbour_list_forms_agree(eng, gab, W):
    """Neighbour lists built with a warp per atom and with a thread per atom
    are the same entry for entry, so every output is bitwise equal (periodic
    cells of several sizes and a molecule in one batch)."""
    s = W.config_c4(n_struct=12, seed=17) + [W.config_c2()]
    mol = W.abx3_cell()
    s.append({"Z": mol["Z"], "pos": mol["pos"] + 2.0, "lat": None})
    out = {}
    try:
        for v in (1, -1):
            gab.set_option("nei_warp", v)
            out[v] = gab.eval_batch(s, dEdLat=True)
    finally:
        gab.set_option("nei_warp", 0)
    for k in ("energy", "forces", "dEdLat"):
        assert np.array_equal(out[1][k], out[-1][k])


def test_compiled_and_runtime_zeta_kernels_agree(eng, gab, W):
    s = W.config_c4(n_struct=6, seed=16)
    fixed = gab.eval_batch(s, dEdLat=True)
    gab.set_option("runtime_zeta", 1)
    try:
        rt = gab.eval_batch(s, dEdLat=True)
    finally:
        gab.set_option("runtime_zeta", 0)
    assert np.abs(fixed["energy"] - rt["energy"]).max() <= E_REL * np.abs(rt["energy"]).max()
    assert np.abs(fixed["forces"] - rt["forces"]).max() <= F_ABS
    assert np.abs(fixed["dEdLat"] - rt["dEdLat"]).max() <= L_ABS


def test_denser_structure_after_a_sparse_one(eng, W, abx3_model):
    """After a call that counted its lists on the host, hdnnp_eval_batch
    searches once into padded rows sized by the densest atom seen so far.  A
    denser structure (the same cell compressed by 20 %: about twice the
    neighbours) overflows them on the device and the call runs again with
    counted lists: the result equals a fresh context's bitwise and the
    oracle's within the FP64 tolerances."""
    rng = np.random.default_rng(62)
    sparse = W.supercell(W.abx3_cell(), (2, 2, 2))
    sparse["pos"] = sparse["pos"] + rng.normal(0.0, 0.1, sparse["pos"].shape)
    dense = {"Z": sparse["Z"], "pos": sparse["pos"] * 0.8, "lat": sparse["lat"] * 0.8}
    p = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        for _ in range(2):  # the first call counts on the host, the second uses padded rows
            p.energy_and_forces(eng.AtStruct(sparse["Z"], sparse["pos"], sparse["lat"]), dEdLat=True)
        E, F, dl = p.energy_and_forces(eng.AtStruct(dense["Z"], dense["pos"], dense["lat"]), dEdLat=True)
        E2, F2, dl2 = p.energy_and_forces(eng.AtStruct(dense["Z"], dense["pos"], dense["lat"]), dEdLat=True)
    finally:
        p.close()
    q = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        E0, F0, dl0 = q.energy_and_forces(eng.AtStruct(dense["Z"], dense["pos"], dense["lat"]), dEdLat=True)
    finally:
        q.close()
    assert E == E0 == E2
    assert np.array_equal(F, F0) and np.array_equal(F2, F0) and np.array_equal(dl, dl0) and np.array_equal(dl2, dl0)
    check(E, F, dl, abx3_model.eval(dense["Z"], dense["pos"], dense["lat"]))


def test_reverse_index_of_padded_rows(eng, W):
    """A context's second call searches into padded rows and builds the
    reverse index while copying them (the mirrored (jx, jy) column of the
    neighbour's row); the first call counts, fills and searches the whole
    list.  Lists and reverse indices are the same entry for entry, for small
    cells with multiple images, larger cells, molecules (one flat) and a cell
    so small that its search spans more columns than the slab table holds."""
    rng = np.random.default_rng(91)
    structs = W.config_c4(n_struct=10, seed=19)
    blob = W.supercell(W.abx3_cell(), (3, 1, 1))
    structs.append({"Z": blob["Z"], "pos": blob["pos"] + rng.normal(0, 0.05, blob["pos"].shape), "lat": None})
    flat = W.abx3_cell()
    fp = flat["pos"].copy()
    fp[:, 2] = 0.0
    fp[:, :2] += rng.normal(0, 0.3, (len(fp), 2))  # the projection puts two atoms on one spot
    structs.append({"Z": flat["Z"], "pos": fp, "lat": None})
    # a 3.6 Bohr cell: 9 x 9 search columns, more than the slab table holds
    structs.append({"Z": np.array([1, 6], np.int32), "pos": np.array([[0.3, 0.2, 0.1], [1.9, 1.7, 2.0]]),
                    "lat": np.eye(3) * 3.6})
    p = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        p.set_option("small_eval", 0)
        out = []
        for _ in range(2):
            r = p.eval_batch(structs, dEdLat=True)
            n = sum(len(s["Z"]) for s in structs)
            cnt = p.fetch("nei_count", n, np.int32)
            tot = int(cnt.sum())
            out.append((r, p.fetch("nei_index", tot, np.int32), p.fetch("nei_shift", tot, np.int32),
                        p.fetch("nei_rev", tot, np.int32)))
    finally:
        p.close()
    (r0, j0, s0, v0), (r1, j1, s1, v1) = out
    assert np.array_equal(j0, j1) and np.array_equal(s0, s1)
    assert np.array_equal(v0, v1), np.nonzero(v0 != v1)[0][:10]
    for k in ("energy", "forces", "dEdLat"):
        assert np.isfinite(r0[k]).all() and np.array_equal(r0[k], r1[k])
