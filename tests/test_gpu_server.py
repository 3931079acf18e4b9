"""Serving form: device-resident walkers with continuous batching.

Checks, each through the C ABI (hdnnp_server_*):
* EVAL, MC trial/reject and MD steps against the FP64 oracle and against a
  host-side velocity-Verlet loop over the plain entry point
  (hdnnpExample.f90:59-64);
* a walker's results are the same alone and in a mix of walkers whose
  requests arrive while others are on the GPU (bitwise for FP64; within the
  mixed-precision error budget, 1e-6 Ha/atom and 1e-5 Ha/Bohr, for MIXED);
* admission by HBM budget, removal freeing budget, error paths.
"""
import threading

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu

RTOL_E, ATOL_F = 1e-10, 1e-9  # FP64 parity bar against the oracle


@pytest.fixture(scope="module")
def pot(pkg):
    from hdnnp_b200 import engine

    p = engine.Hdnnp.from_runner(ABX3_DIR)
    yield p
    p.close()


@pytest.fixture(scope="module")
def S(pkg):
    from hdnnp_b200 import server

    return server


def small_walkers(W, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        shape = [(1, 1, 1), (2, 1, 1), (1, 2, 2), (2, 2, 1), (2, 2, 2)][k % 5]
        s = W.supercell(W.abx3_cell(), shape)
        s["pos"] = s["pos"] + rng.normal(0.0, 0.1, s["pos"].shape)
        out.append(s)
    return out


def test_eval_and_mc_against_oracle(pot, S, W, abx3_model):
    walkers = small_walkers(W, 3, 11)
    with S.Server(pot, max_batch_atoms=4096, workers=2) as srv:
        ids = [srv.add_walker(s["Z"], s["pos"], s["lat"]) for s in walkers]
        tickets = [srv.submit(w, S.REQ_EVAL) for w in ids]
        for s, t in zip(walkers, tickets):
            E, F, dl, lat_ms = srv.wait(t)
            ref = abx3_model.eval(s["Z"], s["pos"], s["lat"])
            assert abs(E - ref["energy"]) <= RTOL_E * abs(ref["energy"])
            assert np.abs(F - ref["forces"]).max() <= ATOL_F
            assert np.abs(dl - ref["dEdLat"]).max() <= ATOL_F
            assert lat_ms >= 0.0
        # trial move: result matches the oracle at the displaced positions
        w, s = ids[1], walkers[1]
        before, _ = srv.read_walker(w)
        E, F, dl, _ = srv.wait(srv.submit(w, S.REQ_MC_TRIAL, sigma=0.05, seed=7))
        moved, _ = srv.read_walker(w)
        d = moved - before
        assert 0.02 < d.std() < 0.08 and np.abs(d.mean()) < 0.02
        ref = abx3_model.eval(s["Z"], moved, s["lat"])
        assert abs(E - ref["energy"]) <= RTOL_E * abs(ref["energy"])
        assert np.abs(F - ref["forces"]).max() <= ATOL_F
        # reject restores the positions bitwise
        srv.wait(srv.submit(w, S.REQ_MC_REJECT))
        back, _ = srv.read_walker(w)
        assert np.array_equal(back, before)
        # an EVAL after the reject reproduces the first result
        E2, F2, _, _ = srv.wait(srv.submit(w, S.REQ_EVAL))
        ref0 = abx3_model.eval(s["Z"], before, s["lat"])
        assert abs(E2 - ref0["energy"]) <= RTOL_E * abs(ref0["energy"])


def test_md_matches_host_verlet_molecule(pkg, S, W, c1):
    """Methylammonium MD (hdnnpExample.f90:59-64) on the device vs the same
    loop on the host over hdnnp_energy_and_forces."""
    from hdnnp_b200 import engine

    s, m, p0 = c1
    p = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    p.set_option("small_eval", 0)  # the plain calls through the pipeline the server runs (bitwise below)
    dt, nsteps = 20.0, 10
    ats = engine.AtStruct(s["Z"], s["pos"].copy())
    E0, F, _ = p.energy_and_forces(ats)
    x, mom = s["pos"].copy(), p0.copy()
    host = []
    for _ in range(nsteps):
        x = x + mom / m[:, None] * dt + 0.5 * F / m[:, None] * dt ** 2
        Fl = F
        E, F, _ = p.energy_and_forces(engine.AtStruct(s["Z"], x))
        mom = mom + dt / 2.0 * (F + Fl)
        host.append((E, F.copy()))
    with S.Server(p, max_batch_atoms=64, workers=1) as srv:
        w = srv.add_walker(s["Z"], s["pos"], None, masses=m, momenta=p0)
        Ed, Fd, _, _ = srv.wait(srv.submit(w, S.REQ_EVAL))
        assert Ed == E0
        for k in range(nsteps):
            Ed, Fd, _, _ = srv.wait(srv.submit(w, S.REQ_MD_STEP, dt=dt))
            Eh, Fh = host[k]
            # the device integrator contracts to FMA; trajectories agree to rounding
            assert abs(Ed - Eh) <= 1e-9 * abs(Eh)
            assert np.abs(Fd - Fh).max() <= 1e-8
        xd, pd = srv.read_walker(w)
        assert np.abs(xd - x).max() <= 1e-9
        assert np.abs(pd - mom).max() <= 1e-9 * max(1.0, np.abs(mom).max())
    p.close()


def run_sequence(srv, S, w, kinds):
    out = []
    for k, (kind, kw) in enumerate(kinds):
        t = srv.submit(w, kind, **kw)
        out.append(srv.wait(t))
    return out


def sequence():
    return [(1, dict(sigma=0.05, seed=3)), (2, {}), (1, dict(sigma=0.05, seed=4)), (0, {}),
            (3, dict(dt=10.0)), (3, dict(dt=10.0)), (1, dict(sigma=0.02, seed=5))]


@pytest.mark.parametrize("precision", [0, 1])
def test_alone_equals_in_mix(pkg, S, W, abx3_model, precision):
    """The probe walker runs the same request sequence alone and while other
    threads keep submitting for other walkers."""
    from hdnnp_b200 import engine

    pot = engine.Hdnnp.from_runner(ABX3_DIR)
    probe = W.supercell(W.abx3_cell(), (2, 2, 1))
    probe["pos"] = probe["pos"] + np.random.default_rng(21).normal(0, 0.1, probe["pos"].shape)
    m, p0 = W.maxwell_boltzmann(probe["Z"], 300.0, 22)
    seq = [(0, {})] + sequence()

    with S.Server(pot, max_batch_atoms=8192, workers=2, precision=precision) as srv:
        w = srv.add_walker(probe["Z"], probe["pos"], probe["lat"], masses=m, momenta=p0)
        alone = run_sequence(srv, S, w, seq)

    with S.Server(pot, max_batch_atoms=8192, workers=2, precision=precision) as srv:
        others = small_walkers(W, 12, 23)
        oid = [srv.add_walker(s["Z"], s["pos"], s["lat"]) for s in others]
        w = srv.add_walker(probe["Z"], probe["pos"], probe["lat"], masses=m, momenta=p0)
        stop = threading.Event()

        def load(ids, seed):
            rng = np.random.default_rng(seed)
            while not stop.is_set():
                ts = [srv.submit(i, int(rng.integers(0, 2)), sigma=0.03, seed=int(rng.integers(1 << 30)))
                      for i in ids]
                for t in ts:
                    srv.wait(t)

        th = [threading.Thread(target=load, args=(oid[k::2], k)) for k in range(2)]
        for t in th:
            t.start()
        try:
            mixed = run_sequence(srv, S, w, seq)
        finally:
            stop.set()
            for t in th:
                t.join()
        st = srv.stats()
    assert st["mean_batch_requests"] > 1.0, st
    for (Ea, Fa, La, _), (Eb, Fb, Lb, _), (kind, _) in zip(alone, mixed, seq):
        if kind == 2:
            continue
        if precision == 0:
            assert Ea == Eb and np.array_equal(Fa, Fb) and np.array_equal(La, Lb)
        else:
            n = len(probe["Z"])
            assert abs(Ea - Eb) / n <= 1e-6 and np.abs(Fa - Fb).max() <= 1e-5
    # the MIXED walker also stays within its budget of the FP64 oracle
    if precision == 1:
        Ea = alone[0][0]
        ref = abx3_model.eval(probe["Z"], probe["pos"], probe["lat"])
        assert abs(Ea - ref["energy"]) / len(probe["Z"]) <= 1e-6
        assert np.abs(alone[0][1] - ref["forces"]).max() <= 1e-5
    pot.close()


def test_admission_by_hbm_budget(pot, S, W):
    from hdnnp_b200.engine import HdnnpError

    walkers = small_walkers(W, 6, 31)
    probe = S.Server(pot, max_batch_atoms=1024, workers=1, hbm_budget=0)
    ws_bytes = probe.stats()["hbm_charged"]
    probe.close()
    per_walker = [len(s["Z"]) * (6 * 24 + 8 + 4) for s in walkers]
    budget = ws_bytes + sum(per_walker[:3]) + per_walker[3] // 2
    with S.Server(pot, max_batch_atoms=1024, workers=1, hbm_budget=budget) as srv:
        ids = [srv.add_walker(s["Z"], s["pos"], s["lat"]) for s in walkers[:3]]
        with pytest.raises(HdnnpError) as e:
            srv.add_walker(walkers[3]["Z"], walkers[3]["pos"], walkers[3]["lat"])
        assert e.value.code == 3
        assert srv.stats()["hbm_charged"] == ws_bytes + sum(per_walker[:3])
        srv.remove_walker(ids[0])  # frees its budget
        if per_walker[3] <= per_walker[0] + per_walker[3] // 2:
            srv.add_walker(walkers[3]["Z"], walkers[3]["pos"], walkers[3]["lat"])
        # workspace alone above the budget
    with pytest.raises(HdnnpError) as e:
        S.Server(pot, max_batch_atoms=1024, workers=1, hbm_budget=ws_bytes - 1)
    assert e.value.code == 3


def test_errors(pot, S, W):
    from hdnnp_b200.engine import HdnnpError

    s = small_walkers(W, 1, 41)[0]
    with S.Server(pot, max_batch_atoms=64, workers=1) as srv:
        with pytest.raises(HdnnpError):  # larger than the slots
            big = W.supercell(W.abx3_cell(), (2, 2, 2))
            srv.add_walker(big["Z"], big["pos"], big["lat"])
        with pytest.raises(HdnnpError):  # element not in the potential
            srv.add_walker(np.full(12, 8), s["pos"], s["lat"])
        w = srv.add_walker(s["Z"], s["pos"], s["lat"])
        with pytest.raises(HdnnpError):  # MD needs masses
            srv.submit(w, S.REQ_MD_STEP, dt=1.0)
        with pytest.raises(HdnnpError):
            srv.submit(w + 100, S.REQ_EVAL)
        with pytest.raises(HdnnpError):
            srv.submit(w, 9)
        t = srv.submit(w, S.REQ_EVAL)
        srv.wait(t)
        with pytest.raises(HdnnpError):  # consumed ticket
            srv.wait(t)
        srv.remove_walker(w)


def test_poisson_load_and_next_done(pot, S, W):
    """Open- and closed-loop load over MD and MC walkers: continuous batching
    packs several walkers' steps per batch and every step completes.  The
    random-weight potential is stiff: an MD trajectory at 300 K and dt = 0.5
    a.u. becomes non-finite after some 500-800 steps (the same step with
    either neighbour-list form), which a second of saturated load can reach;
    such a walker is restarted from its initial state by the load driver, and
    only that failure is allowed."""
    walkers = small_walkers(W, 16, 51)
    with S.Server(pot, max_batch_atoms=4096, workers=2, precision=1) as srv:
        info = []
        for k, s in enumerate(walkers):
            md = k % 2 == 0
            m, p = W.maxwell_boltzmann(s["Z"], 300.0, k) if md else (None, None)
            init = dict(Z=s["Z"], pos=s["pos"], lat=s["lat"], masses=m, momenta=p)
            info.append((srv.add_walker(**init), len(s["Z"]), md, init))
        ts = [srv.submit(w, S.REQ_EVAL) for w, _, _, _ in info]
        seen = set()
        while len(seen) < len(ts):
            t = srv.next_done(10000)
            assert t in ts and t not in seen
            seen.add(t)
            srv.wait(t, 0)
        assert srv.next_done(0) is None
        srv.stats(reset=True)
        sat = S.poisson_load(srv, info, rate=None, duration=1.0, seed=1, dt=0.5)
        assert sat["steps"] > 16 and sat["p99_ms"] >= sat["p50_ms"] > 0
        for wid, msg in sat["failed_walkers"]:
            assert "non-finite position" in msg
        assert srv.stats()["mean_batch_requests"] > 1.0
        opn = S.poisson_load(srv, info, rate=100.0, duration=1.0, seed=2, dt=0.5)
        assert 30 < opn["steps"] < 300
        assert opn["client_p50_ms"] >= opn["p50_ms"] * 0.99


def test_failing_walker_fails_alone(pot, S, W, abx3_model):
    """An MD step whose time step overflows the positions (host-side input
    error; the wrap kernel flags the atoms and keeps every index in bounds)
    fails only that walker's request; the walkers batched with it get their
    results."""
    from hdnnp_b200.engine import HdnnpError

    walkers = small_walkers(W, 4, 61)
    m, p = W.maxwell_boltzmann(walkers[0]["Z"], 300.0, 3)
    with S.Server(pot, max_batch_atoms=8192, workers=1) as srv:
        bad = srv.add_walker(walkers[0]["Z"], walkers[0]["pos"], walkers[0]["lat"], masses=m, momenta=p)
        good = [srv.add_walker(s["Z"], s["pos"], s["lat"]) for s in walkers[1:]]
        srv.wait(srv.submit(bad, S.REQ_EVAL))  # non-zero forces: F/(2m) dt^2 overflows below
        big = W.supercell(W.abx3_cell(), (4, 4, 4))
        busy = srv.add_walker(big["Z"], big["pos"], big["lat"])
        t_busy = srv.submit(busy, S.REQ_EVAL)  # occupies the worker while the next ones queue up
        t_good = [srv.submit(good[0], S.REQ_EVAL)]
        t_bad = srv.submit(bad, S.REQ_MD_STEP, dt=1e300)
        t_good += [srv.submit(w, S.REQ_EVAL) for w in good[1:]]
        srv.wait(t_busy)
        with pytest.raises(HdnnpError) as e:
            srv.wait(t_bad)
        assert e.value.code == 1 and "non-finite" in str(e.value)
        for s, t in zip(walkers[1:], t_good):
            E, F, dl, _ = srv.wait(t)
            ref = abx3_model.eval(s["Z"], s["pos"], s["lat"])
            assert abs(E - ref["energy"]) <= RTOL_E * abs(ref["energy"])
            assert np.abs(F - ref["forces"]).max() <= ATOL_F
        assert srv.stats()["mean_batch_requests"] > 1.0


def test_skin_lists_match_rebuilt_lists(pot, S, W):
    """Walkers that keep their neighbour lists (skin 1 Bohr) follow the same
    trajectories as walkers whose lists are rebuilt for every request (FP64,
    within summation-order rounding), in batches that mix walkers keeping
    and rebuilding lists: MD walkers move little per step and keep theirs,
    Monte Carlo trials of sigma 0.6 Bohr every third step force rebuilds."""
    walkers = small_walkers(W, 6, 61)
    mol = W.abx3_cell()
    walkers.append({"Z": mol["Z"], "pos": mol["pos"] + 4.0, "lat": None})
    kw = dict(max_batch_atoms=4096, workers=1, precision=0)
    with S.Server(pot, **kw) as a, S.Server(pot, skin=1.0, **kw) as b:
        ids = []
        for k, s in enumerate(walkers):
            md = k % 2 == 0
            m, p = W.maxwell_boltzmann(s["Z"], 300.0, 70 + k) if md else (None, None)
            ids.append((a.add_walker(s["Z"], s["pos"], s["lat"], masses=m, momenta=p),
                        b.add_walker(s["Z"], s["pos"], s["lat"], masses=m, momenta=p), md))
        evals = 0
        for step in range(10):
            ta, tb = [], []
            for k, (wa, wb, md) in enumerate(ids):
                if step == 0:
                    args = dict(kind=S.REQ_EVAL)
                elif md:
                    args = dict(kind=S.REQ_MD_STEP, dt=0.5)
                else:
                    args = dict(kind=S.REQ_MC_TRIAL, sigma=0.6 if step % 3 == 0 else 0.02, seed=1000 * step + k)
                ta.append(a.submit(wa, **args))
                tb.append(b.submit(wb, **args))
            for x, y in zip(ta, tb):
                Ea, Fa, La, _ = a.wait(x)
                Eb, Fb, Lb, _ = b.wait(y)
                assert abs(Ea - Eb) <= 1e-10 * abs(Ea)
                assert np.abs(Fa - Fb).max() <= 1e-9
                assert np.abs(La - Lb).max() <= 1e-9
                evals += 1
        st = b.list_stats()
        print("skin lists:", st, "evaluations", evals)
        assert st["built"] + st["kept"] == evals
        assert st["kept"] > 0 and len(walkers) < st["built"] < evals
        assert a.list_stats() == {"built": 0, "kept": 0}


def test_denser_walker_than_the_padded_rows(pot, S, W, abx3_model):
    """Batches that build their lists search once into padded rows sized by
    the densest batch a worker has counted so far.  A walker denser than that
    (the same cell compressed by 20 %: about twice the neighbours) overflows
    the rows on the device; the batch is evaluated again with its counts read
    on the host, and the result matches the oracle and a server that has seen
    nothing sparser."""
    rng = np.random.default_rng(61)
    sparse = W.supercell(W.abx3_cell(), (2, 2, 2))
    sparse["pos"] = sparse["pos"] + rng.normal(0.0, 0.1, sparse["pos"].shape)
    dense = {"Z": sparse["Z"], "pos": sparse["pos"] * 0.8, "lat": sparse["lat"] * 0.8}
    with S.Server(pot, max_batch_atoms=4096, workers=1) as srv:
        a = srv.add_walker(sparse["Z"], sparse["pos"], sparse["lat"])
        for _ in range(2):  # the first batch counts on the host, the second uses padded rows
            srv.wait(srv.submit(a, S.REQ_EVAL))
        b = srv.add_walker(dense["Z"], dense["pos"], dense["lat"])
        E, F, dl, _ = srv.wait(srv.submit(b, S.REQ_EVAL))
        E2, F2, dl2, _ = srv.wait(srv.submit(b, S.REQ_EVAL))  # padded rows now sized for it
    with S.Server(pot, max_batch_atoms=4096, workers=1) as fresh:
        c = fresh.add_walker(dense["Z"], dense["pos"], dense["lat"])
        E0, F0, dl0, _ = fresh.wait(fresh.submit(c, S.REQ_EVAL))
    assert E == E0 == E2 and np.array_equal(F, F0) and np.array_equal(F2, F0) and np.array_equal(dl, dl0)
    ref = abx3_model.eval(dense["Z"], dense["pos"], dense["lat"])
    assert abs(E - ref["energy"]) <= RTOL_E * abs(ref["energy"])
    assert np.abs(F - ref["forces"]).max() <= ATOL_F
