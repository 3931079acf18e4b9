"""The plain entry point on small molecules: one FP64 molecule of at most 64
atoms per call (the reference's MD example calls hdnnpEnergyAndForces this
way, hdnnpExample.f90:58-63) runs as one single-block kernel launch in
evaluation mode, between one copy in and one copy out.

* Equal to the general pipeline (option small_eval 0) within rounding and to
  the FP64 oracle within the FP64 tolerances (|dE| <= 1e-10 |E|, max |dF| <=
  1e-9 Ha/Bohr), for 1 to 64 atoms, both forms of the kernel (item-parallel
  up to ~14 atoms, warp per atom above);
* at most one kernel launch per call (none when the context's resident
  kernel serves it); 65 atoms, periodic cells and the mixed precision use
  the pipeline;
* the resident kernel: bitwise the launched kernel's results, replaced when
  the molecule's size changes or after it left while idle;
* non-finite positions and unknown elements are status codes and the context
  stays usable.
"""
import os

import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu

E_REL, F_ABS = 1e-10, 1e-9


@pytest.fixture(scope="module")
def eng(pkg):
    from hdnnp_b200 import engine

    return engine


def clusters(W):
    rng = np.random.default_rng(81)
    blob = W.supercell(W.abx3_cell(), (2, 2, 2))
    pos = blob["pos"] + rng.normal(0.0, 0.05, blob["pos"].shape)
    out = []
    for n in (1, 2, 5, 13, 31, 60, 64):
        # the n atoms nearest the centre of the 96-atom block
        d = np.linalg.norm(pos - pos.mean(axis=0), axis=1)
        k = np.sort(np.argsort(d)[:n])
        out.append({"Z": blob["Z"][k], "pos": pos[k], "lat": None})
    return out


def test_small_molecules_single_kernel(eng, W, orc, c1):
    cases = [(EXAMPLE_DIR, c1[0])] + [(ABX3_DIR, m) for m in clusters(W)]
    pots = {d: eng.Hdnnp.from_runner(d) for d in (EXAMPLE_DIR, ABX3_DIR)}
    ref_pots = {d: eng.Hdnnp.from_runner(d) for d in (EXAMPLE_DIR, ABX3_DIR)}
    try:
        for p in ref_pots.values():
            p.set_option("small_eval", 0)
        for d, s in cases:
            ats = eng.AtStruct(s["Z"], s["pos"])
            E, F, _ = pots[d].energy_and_forces(ats)
            assert pots[d].launches() <= 1, len(s["Z"])  # 0: the resident kernel served it
            E0, F0, _ = ref_pots[d].energy_and_forces(ats)
            assert ref_pots[d].launches() > 1
            assert abs(E - E0) <= 1e-12 * max(1.0, abs(E0)), (len(s["Z"]), E, E0)
            assert np.abs(F - F0).max() <= 1e-11, len(s["Z"])
            if len(s["Z"]) < 5:
                # the oracle searches every cell of the molecule's box like the
                # reference: for one or two atoms the box is (nearly) flat and
                # that search has ~10^10 cells; the pipeline above is the check
                continue
            ref = orc.Model(d).eval(s["Z"], s["pos"])
            assert abs(E - ref["energy"]) <= E_REL * abs(ref["energy"])
            assert np.abs(F - ref["forces"]).max() <= F_ABS
    finally:
        for p in list(pots.values()) + list(ref_pots.values()):
            p.close()


def test_small_path_boundaries_and_errors(eng, W, c1):
    pot = eng.Hdnnp.from_runner(ABX3_DIR)
    try:
        blob = W.supercell(W.abx3_cell(), (2, 2, 2))
        big = {"Z": blob["Z"][:65], "pos": blob["pos"][:65] + 0.01}
        pot.energy_and_forces(eng.AtStruct(big["Z"], big["pos"]))
        assert pot.launches() > 1  # 65 atoms: the pipeline
        cell = W.abx3_cell()
        pot.energy_and_forces(eng.AtStruct(cell["Z"], cell["pos"], cell["lat"]))
        assert pot.launches() > 1  # periodic: the pipeline
        pot.set_precision(eng.HDNNP_PREC_MIXED)
        pot.energy_and_forces(eng.AtStruct(cell["Z"], cell["pos"]))
        assert pot.launches() > 1  # mixed precision: the pipeline
        pot.set_precision(eng.HDNNP_PREC_FP64)
        mol = {"Z": cell["Z"], "pos": cell["pos"].copy()}
        mol["pos"][3, 2] = np.inf
        with pytest.raises(eng.HdnnpError, match="non-finite"):
            pot.energy_and_forces(eng.AtStruct(mol["Z"], mol["pos"]))
        Z = cell["Z"].copy()
        Z[1] = 8
        with pytest.raises(eng.HdnnpError, match="not in the potential"):
            pot.energy_and_forces(eng.AtStruct(Z, cell["pos"]))
        E, F, _ = pot.energy_and_forces(eng.AtStruct(cell["Z"], cell["pos"]))
        assert np.isfinite(E) and pot.launches() <= 1
    finally:
        pot.close()


def test_resident_kernel_serves_calls(eng, c1):
    """The resident single-block kernel (option small_resident, default on):
    bitwise the results of the launched kernel (option 0); a change of
    molecule size replaces it; after it has left on its own (idle) the next
    call starts another; a non-finite position is an error and the next call
    is served; freeing the context while it waits returns."""
    import time

    ex = c1[0]
    ats = eng.AtStruct(ex["Z"], ex["pos"])
    small = eng.AtStruct(ex["Z"][:5], ex["pos"][:5])
    pot = eng.Hdnnp.from_runner(EXAMPLE_DIR)
    ref = eng.Hdnnp.from_runner(EXAMPLE_DIR)
    try:
        ref.set_option("small_resident", 0)
        E0, F0, _ = ref.energy_and_forces(ats)
        assert ref.launches() == 1
        Es0, Fs0, _ = ref.energy_and_forces(small)
        counts = []
        for k in range(6):
            s = ats if k % 3 != 2 else small
            E, F, _ = pot.energy_and_forces(s)
            counts.append(pot.launches())
            if s is ats:
                assert E == E0 and np.array_equal(F, F0)
            else:
                assert E == Es0 and np.array_equal(F, Fs0)
        # launched on the first call and after each change of size; the calls
        # in between are served by the running kernel (a host pause of more
        # than a few milliseconds would let it leave, hence "or")
        assert counts[0] == counts[2] == counts[3] == counts[5] == 1, counts
        assert counts[1] == 0 or counts[4] == 0, counts
        time.sleep(0.05)  # idle: the kernel leaves after a few milliseconds
        E, F, _ = pot.energy_and_forces(ats)
        assert pot.launches() == 1 and E == E0 and np.array_equal(F, F0)
        bad = ex["pos"].copy()
        bad[2, 1] = np.nan
        with pytest.raises(eng.HdnnpError):
            pot.energy_and_forces(eng.AtStruct(ex["Z"], bad))
        E, F, _ = pot.energy_and_forces(ats)
        assert E == E0 and np.array_equal(F, F0)
        # switched off: the launched kernel again
        pot.set_option("small_resident", 0)
        E, F, _ = pot.energy_and_forces(ats)
        assert pot.launches() == 1 and E == E0 and np.array_equal(F, F0)
        pot.set_option("small_resident", 1)
        pot.energy_and_forces(ats)
    finally:
        t0 = time.perf_counter()
        pot.close()  # the resident kernel is waiting: freeing the context stops it
        assert time.perf_counter() - t0 < 1.0
        ref.close()
