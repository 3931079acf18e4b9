"""hdnnp_energy_and_forces_noalloc against hdnnp_energy_and_forces.

The no-allocation entry point serves callers that cannot allocate GPU memory
at evaluation time (an MD or Monte Carlo host code under a fixed device-memory
budget handed out at start-up, bindings without the CUDA allocator): it keeps
every intermediate in one static device array.  This test calls it through
the C ABI twice in a row on the same inputs (the array keeps the previous
call's contents) and compares each result with the context-based entry point,
and once with the FP64 oracle, with the FP64 tolerances used by the other
parity tests.  It also checks the capacity limits and argument errors, and
that a context evaluation on the same device is unaffected after each
failure.  It lives in its own file so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu

E_REL, F_ABS, L_ABS = 1e-10, 1e-9, 1e-9


def _noalloc(eng, pot, s, want_dEdLat):
    L = eng.lib()
    fn = L.hdnnp_energy_and_forces_noalloc
    fn.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int,
                   C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    Z = np.ascontiguousarray(s["Z"], dtype=np.int32)
    pos = np.ascontiguousarray(s["pos"], dtype=np.float64)
    per = s["lat"] is not None
    lat = np.asarray(s["lat"], dtype=np.float64).ravel(order="F").copy() if per else None
    E = C.c_double()
    F = np.zeros((len(Z), 3))
    dl = np.zeros(9) if want_dEdLat else None
    dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
    code = fn(pot._m, len(Z), Z.ctypes.data_as(C.POINTER(C.c_int32)), dp(pos), 1 if per else 0, dp(lat),
              C.byref(E), dp(F), dp(dl))
    if code != 0:
        raise eng.HdnnpError(code, L.hdnnp_last_error().decode())
    return E.value, F, (dl.reshape(3, 3, order="F") if dl is not None else None)


def _cases(W):
    rng = np.random.default_rng(21)
    cell = W.strain(W.abx3_cell(), rng.uniform(-0.05, 0.05, (3, 3)))
    cell["pos"] = cell["pos"] + rng.normal(0, 0.15, cell["pos"].shape)
    return [("example", EXAMPLE_DIR, W.read_xyz(EXAMPLE_DIR + "/input.xyz"), False),
            ("cell12", ABX3_DIR, cell, True),
            ("cell768", ABX3_DIR, W.config_c2(seed=9), True)]


def test_noalloc_matches_context_entry_point_twice(pkg, W):
    from hdnnp_b200 import engine as eng

    for name, d, s, stress in _cases(W):
        pot = eng.Hdnnp.from_runner(d)
        try:
            ats = eng.AtStruct(s["Z"], s["pos"], s["lat"])
            E0, F0, L0 = pot.energy_and_forces(ats, dEdLat=stress)
            for call in range(2):
                E1, F1, L1 = _noalloc(eng, pot, s, stress)
                assert abs(E1 - E0) <= E_REL * abs(E0), (name, call, E1, E0)
                assert np.abs(F1 - F0).max() <= F_ABS, (name, call)
                if stress:
                    assert np.abs(L1 - L0).max() <= L_ABS, (name, call)
        finally:
            pot.close()


def test_noalloc_rejects_structures_beyond_the_scratch(pkg, W):
    from hdnnp_b200 import engine as eng

    pot = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        big = W.supercell(W.abx3_cell(), (8, 8, 8))  # 6,144 atoms
        big = W.supercell(big, (2, 1, 1))            # 12,288 atoms: more than 32 MiB of intermediates
        with pytest.raises(eng.HdnnpError, match="static scratch"):
            _noalloc(eng, pot, big, True)
        # still usable afterwards
        s = W.config_c2(seed=3)
        E0, _, _ = pot.energy_and_forces(eng.AtStruct(s["Z"], s["pos"], s["lat"]))
        E1, _, _ = _noalloc(eng, pot, s, False)
        assert abs(E1 - E0) <= E_REL * abs(E0)
    finally:
        pot.close()


def test_noalloc_matches_the_oracle(pkg, W, orc):
    from hdnnp_b200 import engine as eng

    s = W.config_c2(seed=11)
    pot = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        E1, F1, L1 = _noalloc(eng, pot, s, True)
    finally:
        pot.close()
    ref = orc.Model(ABX3_DIR).eval(s["Z"], s["pos"], s["lat"])
    assert abs(E1 - ref["energy"]) <= E_REL * abs(ref["energy"])
    assert np.abs(F1 - ref["forces"]).max() <= F_ABS
    assert np.abs(L1 - ref["dEdLat"]).max() <= L_ABS


def _context_still_right(eng, pot, s, orc_model):
    E, F, _ = pot.energy_and_forces(eng.AtStruct(s["Z"], s["pos"], s["lat"]))
    ref = orc_model.eval(s["Z"], s["pos"], s["lat"])
    assert abs(E - ref["energy"]) <= E_REL * abs(ref["energy"])
    assert np.abs(F - ref["forces"]).max() <= F_ABS


def test_noalloc_entry_overflow_and_argument_errors(pkg, W, orc):
    """A dense 2,000-atom cluster fits the per-atom arrays of the static
    scratch but not its neighbour entries (~1,000 per atom); bad arguments
    are refused before any device work.  A context evaluation on the same
    device gives the oracle's result after each failure."""
    from hdnnp_b200 import engine as eng

    rng = np.random.default_rng(31)
    n = 2000
    d = rng.normal(size=(n, 3))
    ball = d / np.linalg.norm(d, axis=1)[:, None] * (11.0 * rng.uniform(size=(n, 1)) ** (1 / 3))
    dense = {"Z": rng.choice(np.array([1, 6, 7, 53, 82], dtype=np.int32), n), "pos": ball, "lat": None}
    good = W.config_c2(seed=5)
    om = orc.Model(ABX3_DIR)
    pot = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        with pytest.raises(eng.HdnnpError, match="too many neighbour entries") as ei:
            _noalloc(eng, pot, dense, False)
        assert ei.value.code == 3
        _context_still_right(eng, pot, good, om)
        mol = W.read_xyz(EXAMPLE_DIR + "/input.xyz")
        mol_ab = {"Z": np.array([6, 7, 1, 1], dtype=np.int32), "pos": mol["pos"][:4], "lat": None}
        with pytest.raises(eng.HdnnpError, match="periodic") as ei:
            _noalloc(eng, pot, mol_ab, True)  # dEdLat of a molecule
        assert ei.value.code == 1
        _context_still_right(eng, pot, good, om)
        L = eng.lib()
        fn = L.hdnnp_energy_and_forces_noalloc
        Z = np.ascontiguousarray(good["Z"], dtype=np.int32)
        pos = np.ascontiguousarray(good["pos"])
        E = C.c_double()
        F = np.zeros((len(Z), 3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        code = fn(pot._m, len(Z), Z.ctypes.data_as(C.POINTER(C.c_int32)), dp(pos), 1, None, C.byref(E), dp(F), None)
        assert code == 1 and "lattice" in L.hdnnp_last_error().decode()
        _context_still_right(eng, pot, good, om)
        badZ = dict(good, Z=np.where(np.arange(len(Z)) == 7, 8, good["Z"]).astype(np.int32))  # oxygen
        with pytest.raises(eng.HdnnpError, match="Z=8") as ei:
            _noalloc(eng, pot, badZ, False)
        assert ei.value.code == 1
        _context_still_right(eng, pot, good, om)
        # and the no-allocation path itself still evaluates correctly
        E1, F1, _ = _noalloc(eng, pot, good, False)
        ref = om.eval(good["Z"], good["pos"], good["lat"])
        assert abs(E1 - ref["energy"]) <= E_REL * abs(ref["energy"])
        assert np.abs(F1 - ref["forces"]).max() <= F_ABS
    finally:
        pot.close()
