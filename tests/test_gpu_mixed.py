"""Mixed-precision form (FP32 symmetry functions and networks; FP64 wrap,
energy sum and virial reduction) against the FP64 oracle.

Error budget of the north star, stated here and asserted:
  |dE| per atom <= 1e-6 Ha, max |dF| <= 1e-5 Ha/Bohr, and dE/dh per atom
  <= 1e-5 Ha/Bohr.  Every test prints the measured errors.
"""
import numpy as np
import pytest

from conftest import ABX3_DIR, EXAMPLE_DIR

pytestmark = pytest.mark.gpu

E_ATOM, F_ABS, L_ATOM = 1e-6, 1e-5, 1e-5


@pytest.fixture(scope="module")
def gmix(pkg):
    from hdnnp_b200 import engine

    p = engine.Hdnnp.from_runner(ABX3_DIR)
    p.set_precision(engine.HDNNP_PREC_MIXED)
    yield p
    p.close()


def errors(out, structs, model):
    off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
    eE, eF, eL = 0.0, 0.0, 0.0
    for k, s in enumerate(structs):
        ref = model.eval(s["Z"], s["pos"], s["lat"])
        n = len(s["Z"])
        eE = max(eE, abs(out["energy"][k] - ref["energy"]) / n)
        eF = max(eF, np.abs(out["forces"][off[k]:off[k + 1]] - ref["forces"]).max())
        if s["lat"] is not None:
            dl = out["dEdLat"][9 * k:9 * k + 9].reshape(3, 3, order="F")
            eL = max(eL, np.abs(dl - ref["dEdLat"]).max() / n)
    return eE, eF, eL


def test_mixed_768_atoms(gmix, abx3_model, W):
    s = [W.config_c2()]
    eE, eF, eL = errors(gmix.eval_batch(s, dEdLat=True), s, abx3_model)
    print(f"mixed 768 atoms: |dE|/atom {eE:.2e}  max|dF| {eF:.2e}  |d dEdLat|/atom {eL:.2e}")
    assert eE <= E_ATOM and eF <= F_ABS and eL <= L_ATOM


def test_mixed_batch(gmix, abx3_model, W):
    s = W.config_c4(n_struct=24, seed=14)
    eE, eF, eL = errors(gmix.eval_batch(s, dEdLat=True), s, abx3_model)
    print(f"mixed batch: |dE|/atom {eE:.2e}  max|dF| {eF:.2e}  |d dEdLat|/atom {eL:.2e}")
    assert eE <= E_ATOM and eF <= F_ABS and eL <= L_ATOM


def test_mixed_example_molecule(pkg, ex_model, c1):
    from hdnnp_b200 import engine

    p = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    p.set_precision(engine.HDNNP_PREC_MIXED)
    s = c1[0]
    E, F, _ = p.energy_and_forces(engine.AtStruct(s["Z"], s["pos"]))
    ref = ex_model.eval(s["Z"], s["pos"])
    p.close()
    print(f"mixed example: |dE|/atom {abs(E - ref['energy']) / 8:.2e}  max|dF| {np.abs(F - ref['forces']).max():.2e}")
    assert abs(E - ref["energy"]) / 8 <= E_ATOM
    assert np.abs(F - ref["forces"]).max() <= F_ABS


def test_mixed_alone_equals_in_mix(gmix, W):
    structs = W.config_c4(n_struct=12, seed=15)
    mix = gmix.eval_batch(structs, dEdLat=True)
    off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
    for k in (0, 7, 11):
        alone = gmix.eval_batch([structs[k]], dEdLat=True)
        assert abs(alone["energy"][0] - mix["energy"][k]) <= 1e-9 * len(structs[k]["Z"])
        assert np.abs(alone["forces"] - mix["forces"][off[k]:off[k + 1]]).max() <= 1e-9


def test_tensor_core_network_matches_simt(gmix, W):
    """tcgen05 FP16 hi+lo network (default) vs the FP32 CUDA-core network."""
    s = W.config_c4(n_struct=10, seed=17)
    tc = gmix.eval_batch(s, dEdLat=True)
    gmix.set_option("mlp_simt", 1)
    try:
        simt = gmix.eval_batch(s, dEdLat=True)
    finally:
        gmix.set_option("mlp_simt", 0)
    nat = np.array([len(x["Z"]) for x in s])
    dE = np.abs(tc["energy"] - simt["energy"]) / nat
    dF = np.abs(tc["forces"] - simt["forces"]).max()
    print(f"tensor-core vs SIMT network: |dE|/atom {dE.max():.2e}  max|dF| {dF:.2e}")
    assert dE.max() <= 1e-6 and dF <= 1e-5
