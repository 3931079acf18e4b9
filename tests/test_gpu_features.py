"""Reference features that the example and ABX3 potentials leave out, on the
GPU against the FP64 oracle (potential tests/golden/prz, made by
tests/golden/make_prz_potential.py):

* softplus and ReLU layers (activate / deactivate,
  neuralNetworks.f90:45-49 and :69-80), as "p r l" and, from a copy with the
  activation line changed, "r p t";
* angular functions with non-integer zeta 2.5 and 6.3 (the real-power branch
  of calcAllSymmetryFunctions, symmetryFunctions.f90:266-273), evaluated by
  the lambda x zeta x eta kernels with the zeta set read from the model (the
  power by pow()) and by the generic kernels (one record per function).

FP64: |dE| <= 1e-10 |E|, max |dF| and max |d dE/dh| <= 1e-9.  Mixed: |dE|
per atom <= 1e-6, max |dF| <= 1e-5, |d dE/dh| per atom <= 1e-5.
"""
import os
import shutil

import numpy as np
import pytest

from conftest import EXAMPLE_DIR, PRZ_DIR

pytestmark = pytest.mark.gpu

E_REL, F_ABS, L_ABS = 1e-10, 1e-9, 1e-9
E_ATOM, F_MIX, L_ATOM = 1e-6, 1e-5, 1e-5


@pytest.fixture(scope="module")
def eng(pkg):
    from hdnnp_b200 import engine

    return engine


@pytest.fixture(scope="module")
def rpt_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("rpt")
    for f in os.listdir(PRZ_DIR):
        shutil.copy(os.path.join(PRZ_DIR, f), d / f)
    txt = (d / "input.nn").read_text()
    assert "global_activation_short p r l" in txt
    (d / "input.nn").write_text(txt.replace("global_activation_short p r l", "global_activation_short r p t"))
    return str(d)


def structures(W):
    rng = np.random.default_rng(61)
    out = []
    for shape in ((1, 1, 1), (2, 1, 1), (2, 2, 2)):
        c = W.strain(W.supercell(W.abx3_cell(), shape), rng.uniform(-0.05, 0.05, (3, 3)))
        c["pos"] = c["pos"] + rng.normal(0, 0.15, c["pos"].shape)
        out.append(c)
    out.append(W.config_c2(seed=62))
    mol = W.read_xyz(os.path.join(EXAMPLE_DIR, "input.xyz"))  # C, N, H: elements of this potential
    out.append(mol)
    return out


def run_and_check(eng, path, orc, W, precision, generic=False, simt=False):
    pot = eng.Hdnnp.from_runner(path)
    model = orc.Model(path)
    structs = structures(W) + W.config_c4(n_struct=10, seed=63)
    worst = [0.0, 0.0, 0.0]
    try:
        pot.set_precision(precision)
        if generic:
            pot.set_option("generic_sf", 1)
        if simt:
            pot.set_option("mlp_simt", 1)
        for s in structs:
            per = s["lat"] is not None
            E, F, dl = pot.energy_and_forces(eng.AtStruct(s["Z"], s["pos"], s["lat"]), dEdLat=per)
            ref = model.eval(s["Z"], s["pos"], s["lat"])
            n = len(s["Z"])
            if precision == eng.HDNNP_PREC_FP64:
                errs = (abs(E - ref["energy"]) / abs(ref["energy"]), np.abs(F - ref["forces"]).max(),
                        np.abs(dl - ref["dEdLat"]).max() if per else 0.0)
                lim = (E_REL, F_ABS, L_ABS)
            else:
                errs = (abs(E - ref["energy"]) / n, np.abs(F - ref["forces"]).max(),
                        np.abs(dl - ref["dEdLat"]).max() / n if per else 0.0)
                lim = (E_ATOM, F_MIX, L_ATOM)
            worst = [max(a, b) for a, b in zip(worst, errs)]
            assert all(e <= l for e, l in zip(errs, lim)), (n, errs)
        # the batched form of the same structures
        out = pot.eval_batch(structs, dEdLat=True)
        off = np.concatenate([[0], np.cumsum([len(s["Z"]) for s in structs])])
        for k, s in enumerate(structs):
            ref = model.eval(s["Z"], s["pos"], s["lat"])
            tol = F_ABS if precision == eng.HDNNP_PREC_FP64 else F_MIX
            assert np.abs(out["forces"][off[k]:off[k + 1]] - ref["forces"]).max() <= tol
    finally:
        pot.close()
    return worst


@pytest.mark.parametrize("generic", [False, True])
def test_softplus_relu_noninteger_zeta_fp64(eng, orc, W, generic):
    w = run_and_check(eng, PRZ_DIR, orc, W, eng.HDNNP_PREC_FP64, generic=generic)
    print(f"p r l, zeta 1/2.5/6.3, FP64 ({'generic' if generic else 'lambda x zeta x eta'} kernels): "
          f"|dE|/|E| {w[0]:.2e}  max|dF| {w[1]:.2e}  max|d dEdLat| {w[2]:.2e}")


@pytest.mark.parametrize("simt", [False, True])
def test_softplus_relu_noninteger_zeta_mixed(eng, orc, W, simt):
    w = run_and_check(eng, PRZ_DIR, orc, W, eng.HDNNP_PREC_MIXED, simt=simt)
    print(f"p r l, zeta 1/2.5/6.3, mixed ({'SIMT' if simt else 'tensor-core'} network): "
          f"|dE|/atom {w[0]:.2e}  max|dF| {w[1]:.2e}  |d dEdLat|/atom {w[2]:.2e}")


def test_relu_softplus_tanh_output(eng, orc, W, rpt_dir):
    w64 = run_and_check(eng, rpt_dir, orc, W, eng.HDNNP_PREC_FP64)
    wmx = run_and_check(eng, rpt_dir, orc, W, eng.HDNNP_PREC_MIXED)
    print(f"r p t: FP64 |dE|/|E| {w64[0]:.2e} max|dF| {w64[1]:.2e}; mixed |dE|/atom {wmx[0]:.2e} max|dF| {wmx[1]:.2e}")


def test_single_block_md_with_softplus_relu(pkg, eng, orc, W):
    """The single-block MD kernel of small molecules follows the graph of
    separate kernels with these activations and zeta values too, and its
    forces equal the oracle's at its final positions."""
    from hdnnp_b200 import plan as PL

    mol = W.read_xyz(os.path.join(EXAMPLE_DIR, "input.xyz"))
    m, p0 = W.maxwell_boltzmann(mol["Z"], 140.0, 64)
    pot = eng.Hdnnp.from_runner(PRZ_DIR)
    model = orc.Model(PRZ_DIR)
    try:
        kw = dict(masses=m, momenta=p0, dt=10.0, steps_per_launch=9, want_dEdLat=False)
        with PL.Plan(pot, [mol], **kw) as a, PL.Plan(pot, [mol], single_block=False, **kw) as b:
            assert a.info()["kernels_per_launch"] == 1
            for _ in range(2):
                a.launch()
                b.launch()
                a.sync()
                b.sync()
            assert np.abs(a.F.cpu().numpy() - b.F.cpu().numpy()).max() <= 1e-8
            pos = a.pos.cpu().numpy()
            ref = model.eval(mol["Z"], pos)
            assert np.abs(a.F.cpu().numpy() - ref["forces"]).max() <= F_ABS
            assert abs(a.E.cpu().numpy()[0] - ref["energy"]) <= E_REL * abs(ref["energy"])
    finally:
        pot.close()
