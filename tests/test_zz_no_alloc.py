"""hdnnp_energy_and_forces_noalloc against hdnnp_energy_and_forces.

The no-allocation entry point serves callers that cannot allocate GPU memory
at evaluation time (fixed device-memory budgets, evaluation inside someone
else's stream capture, bindings without the CUDA allocator): it keeps every
intermediate in one static device array.  This test calls it through the C
ABI twice in a row on the same inputs (the array keeps the previous call's
contents) and compares each result with the context-based entry point, with
the FP64 tolerances used by the other parity tests.  It lives in its own file
so that pytest collects it last.
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
