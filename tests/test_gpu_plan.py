"""Resident plans (CUDA-graph evaluations, device-side MD, Verlet-skin lists).

* A plan's evaluation equals the eager batched evaluation bitwise (FP64), for
  periodic cells and molecules (box built on the device), also after the
  positions change in place.
* An MD plan of the methylammonium example follows the host-side velocity
  Verlet loop of hdnnpExample.f90:59-64 over the plain entry point (to FMA
  rounding).
* Verlet-skin lists (skin 1 Bohr) give the same trajectory as lists rebuilt
  every step, within 1e-10 relative (summation order only), with fewer builds.
* Neighbour counts above the planned capacity are flagged (HDNNP_E_CAPACITY),
  with every access kept inside the reserved arrays.
"""
import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pot(pkg):
    from hdnnp_b200 import engine

    p = engine.Hdnnp.from_runner(ABX3_DIR)
    yield p
    p.close()


@pytest.fixture(scope="module")
def PL(pkg):
    from hdnnp_b200 import plan

    return plan


def cells(W, shapes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for n in shapes:
        s = W.supercell(W.abx3_cell(), n)
        s["pos"] = s["pos"] + rng.normal(0.0, 0.1, s["pos"].shape)
        out.append(s)
    return out


def test_plan_equals_eager_batch(pot, PL, W):
    structs = cells(W, [(1, 1, 1), (2, 1, 1), (2, 2, 2)], 3)
    mol = W.abx3_cell()
    structs.append({"Z": mol["Z"], "pos": mol["pos"] + 3.0, "lat": None})  # a molecule
    ref = pot.eval_batch(structs, dEdLat=True)
    with PL.Plan(pot, structs) as p:
        E0, F0, D0 = p.results()  # the probe evaluation
        p.launch()
        assert p.sync() == 1
        E, F, D = p.results()
        assert np.array_equal(E, ref["energy"]) and np.array_equal(E, E0)
        assert np.array_equal(F, ref["forces"]) and np.array_equal(F, F0)
        assert np.array_equal(D.transpose(0, 2, 1).reshape(-1), ref["dEdLat"])
        # positions changed in place (the molecule's box moves with them)
        rng = np.random.default_rng(4)
        moved = [dict(s, pos=s["pos"] + rng.normal(0, 0.05, s["pos"].shape)) for s in structs]
        import torch

        p.pos.copy_(torch.from_numpy(np.concatenate([s["pos"] for s in moved])))
        p.launch()
        p.sync()
        E, F, D = p.results()
        ref = pot.eval_batch(moved, dEdLat=True)
        assert np.array_equal(E, ref["energy"]) and np.array_equal(F, ref["forces"])


def test_md_plan_matches_host_verlet(pkg, PL, c1):
    from hdnnp_b200 import engine

    s, m, p0 = c1
    pot = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    dt, k, launches = 20.0, 5, 4
    E, F, _ = pot.energy_and_forces(engine.AtStruct(s["Z"], s["pos"]))
    x, mom = s["pos"].copy(), p0.copy()
    host = []
    for _ in range(k * launches):
        x = x + mom / m[:, None] * dt + 0.5 * F / m[:, None] * dt ** 2
        Fl = F
        E, F, _ = pot.energy_and_forces(engine.AtStruct(s["Z"], x))
        mom = mom + dt / 2.0 * (F + Fl)
        host.append(E)
    with PL.Plan(pot, [{"Z": s["Z"], "pos": s["pos"], "lat": None}], masses=m, momenta=p0, dt=dt,
                 steps_per_launch=k, want_dEdLat=False) as p:
        energies = []
        for _ in range(launches):
            p.launch()
            p.sync()
            energies += p.hist.cpu().numpy()[:, 0].tolist()
        _, Fd, _ = p.results()
        xd = p.pos.cpu().numpy()
        pd = p.mom.cpu().numpy()
    assert np.allclose(energies, host, rtol=1e-9, atol=0)
    assert np.abs(Fd - F).max() <= 1e-8
    assert np.abs(xd - x).max() <= 1e-9
    assert np.abs(pd - mom).max() <= 1e-9 * max(1.0, np.abs(mom).max())
    pot.close()


def test_single_block_md_matches_graph(pkg, PL, c1, pot, W):
    """MD of a small molecule in one kernel per launch follows the graph of
    separate kernels (same formulas; other summation orders, so to rounding):
    the item-parallel form for the 8-atom example, a 2-atom fragment of it (no
    angular pairs) and an 8-atom fragment of the ABX3 cell (280 functions per
    element); the warp-per-atom form for a 60-atom ABX3 cluster."""
    from hdnnp_b200 import engine

    s, m, p0 = c1
    ex = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    blob = W.supercell(W.abx3_cell(), (1, 1, 5))  # 60 atoms
    rng = np.random.default_rng(21)
    mol = {"Z": blob["Z"], "pos": blob["pos"] + rng.normal(0.0, 0.05, blob["pos"].shape), "lat": None}
    mm, pm = W.maxwell_boltzmann(mol["Z"], 300.0, 22)
    frag = {"Z": mol["Z"][:8], "pos": mol["pos"][:8], "lat": None}
    two = {"Z": s["Z"][:2], "pos": s["pos"][:2], "lat": None}
    cases = ((ex, {"Z": s["Z"], "pos": s["pos"], "lat": None}, m, p0, 20.0),
             (ex, two, m[:2], p0[:2], 20.0),
             (pot, frag, mm[:8], pm[:8], 0.5),
             (pot, mol, mm, pm, 0.5))
    for model, st, masses, mom, dt in cases:
        kw = dict(masses=masses, momenta=mom, dt=dt, steps_per_launch=7, want_dEdLat=False)
        with PL.Plan(model, [st], **kw) as a, PL.Plan(model, [st], single_block=False, **kw) as b:
            assert a.info()["kernels_per_launch"] == 1 and b.info()["kernels_per_launch"] > 10
            for _ in range(3):
                a.launch()
                b.launch()
                assert a.sync() == 7 and b.sync() == 7
                ea, eb = a.hist.cpu().numpy(), b.hist.cpu().numpy()
                assert np.allclose(ea, eb, rtol=1e-9, atol=0)
            assert np.abs(a.F.cpu().numpy() - b.F.cpu().numpy()).max() <= 1e-8
            assert np.abs(a.pos.cpu().numpy() - b.pos.cpu().numpy()).max() <= 1e-9
            assert np.abs(a.mom.cpu().numpy() - b.mom.cpu().numpy()).max() <= 1e-9 * max(1.0, np.abs(mom).max())
            # a non-finite momentum is flagged like the graph path's check
            a.mom[0, 0] = float("nan")
            a.launch()
            with pytest.raises(engine.HdnnpError):
                a.sync()
    ex.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_skin_lists_match_rebuilt_lists(pot, PL, W, precision):
    s = cells(W, [(2, 2, 2)], 8)[0]
    m, p0 = W.maxwell_boltzmann(s["Z"], 300.0, 9)
    kw = dict(precision=precision, masses=m, momenta=p0, dt=0.5, steps_per_launch=10, want_dEdLat=False)
    with PL.Plan(pot, [s], skin=0.0, **kw) as a, PL.Plan(pot, [s], skin=1.0, **kw) as b:
        builds = 0
        for _ in range(3):
            a.launch()
            b.launch()
            assert a.sync() == 10
            builds += b.sync()
            ea, eb = a.hist.cpu().numpy(), b.hist.cpu().numpy()
            if precision == 0:
                assert np.allclose(ea, eb, rtol=1e-10, atol=0)
            else:
                assert np.abs(ea - eb).max() / len(s["Z"]) <= 1e-6
        Fa, Fb = a.F.cpu().numpy(), b.F.cpu().numpy()
        assert np.abs(Fa - Fb).max() <= (1e-9 if precision == 0 else 1e-5)
        assert builds < 30  # most steps reused the list
        # a uniform shift by more than skin/2 forces a rebuild (and moves the
        # wrap); the energy is translation invariant
        for q in (a, b):
            q.pos.add_(0.6)
        a.launch()
        b.launch()
        a.sync()
        assert b.sync() >= 1
        ea, eb = a.hist.cpu().numpy(), b.hist.cpu().numpy()
        if precision == 0:
            assert np.allclose(ea, eb, rtol=1e-10, atol=0)
        else:
            assert np.abs(ea - eb).max() / len(s["Z"]) <= 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_skin_lists_are_compacted(pot, PL, W, precision):
    """The stages after the list read only the entries of a skin list that lie
    within rc: as many as a list built without the skin, in a cell whose atoms
    moved after the build (kept list), for a batch of cells and a molecule."""
    import torch

    structs = cells(W, [(3, 3, 3), (2, 2, 1)], 21)
    mol = W.abx3_cell()
    structs.append({"Z": mol["Z"], "pos": mol["pos"] + 1.0, "lat": None})
    kw = dict(precision=precision, profile=True)
    with PL.Plan(pot, structs, skin=0.0, **kw) as a, PL.Plan(pot, structs, skin=1.0, **kw) as b:
        rng = np.random.default_rng(4)
        step = torch.from_numpy(rng.normal(0.0, 0.08, tuple(a.pos.shape))).to(a.pos.device)
        for q in (a, b):
            q.launch()
            q.sync()
            q.pos.add_(step)  # |step| < skin/2 for every atom: b keeps its list
            q.profile(reset=True)
            q.launch()
        assert a.sync() == 1 and b.sync() == 0
        ca, cb = a.profile()[1], b.profile()[1]
        assert cb["entries"] == ca["entries"] and cb["pairs"] == ca["pairs"]
        Ea, Fa, _ = a.results()
        Eb, Fb, _ = b.results()
        tol_e, tol_f = (1e-10, 1e-9) if precision == 0 else (1e-6, 1e-5)
        assert np.abs(Ea - Eb).max() <= tol_e * np.abs(Ea).max()
        assert np.abs(Fa - Fb).max() <= tol_f


def test_capacity_overflow_is_flagged(pot, PL, W):
    import torch
    from hdnnp_b200.engine import HdnnpError

    s = cells(W, [(2, 2, 2)], 10)[0]
    with PL.Plan(pot, [s], margin=0.0) as p:
        p.launch()
        p.sync()
        # crowd all atoms into a 2-Bohr ball: ~95 neighbours each, above the plan's capacity
        rng = np.random.default_rng(11)
        ball = 20.0 + rng.uniform(-1.0, 1.0, s["pos"].shape)
        p.pos.copy_(torch.from_numpy(ball))
        p.launch()
        with pytest.raises(HdnnpError) as e:
            p.sync()
        assert e.value.code == 3
        # back to the original positions: the same plan works again
        p.pos.copy_(torch.from_numpy(s["pos"]))
        p.launch()
        p.sync()
        ref = pot.eval_batch([s], dEdLat=False)
        assert np.array_equal(p.results()[0], ref["energy"])


def test_autotuned_plan_equals_eager(pot, PL, W):
    """The autotuner only changes the launch shape of the symmetry-function
    kernels; every shape gives bitwise the same FP64 result."""
    structs = cells(W, [(2, 2, 2), (3, 2, 2), (1, 1, 2)], 13)
    ref = pot.eval_batch(structs, dEdLat=True)
    with PL.Plan(pot, structs, autotune=True) as p:
        t = p.tuning()
        assert t["sf_blocks_per_sm"] in (8, 16, 32) and t["sf_split"] in (-1, 32, 48, 64, 96) and t["sf_ms"] > 0
        p.launch()
        p.sync()
        E, F, D = p.results()
    assert np.array_equal(E, ref["energy"]) and np.array_equal(F, ref["forces"])
    for split in (-1, 32, 96):
        pot.set_option("sf_split", split)
        pot.set_option("sf_blocks_per_sm", 8)
        out = pot.eval_batch(structs, dEdLat=True)
        assert np.array_equal(out["energy"], ref["energy"]) and np.array_equal(out["forces"], ref["forces"])
    pot.set_option("sf_split", 0)
    pot.set_option("sf_blocks_per_sm", 0)
