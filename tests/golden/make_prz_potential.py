"""Generates a small synthetic RuNNer potential that exercises the parts of
the reference the ABX3 and example potentials leave out (tests/golden/prz/):

* softplus and ReLU layers: global_activation_short p r l
  (activate / deactivate, neuralNetworks.f90:45-49 and :69-80);
* angular symmetry functions with non-integer zeta (the real-power branch of
  calcAllSymmetryFunctions, symmetryFunctions.f90:266-273): zeta in
  {1, 2.5, 6.3} x lambda +-1 x eta {0.001, 0.013} (a non-integer eta ratio:
  the FP64 kernels take one exponential per eta) for each of the 15 element
  pairs of H, C, N, I, Pb, plus 3 radial functions per neighbour element
  (eta 0.002, 0.05, 0.4; Rs 0): 15 + 180 = 195 per element, rc 11 Bohr,
  tanh^3 cutoff (cutoff_type 2).

Weights: W ~ N(0, 1/fan_in), b ~ N(0, 1/fan_in), seed 4321, 195-16-12-1.
scaling.data: min/max/mean of every symmetry function over the 768-atom ABX3
cell (seed 1) and 64 structures drawn like the batched workload (seed 45),
from the FP64 oracle on unscaled functions, each range floored at half the
function's largest magnitude (and 1e-6) as for the ABX3 potential.
Run from the repository root:  python tests/golden/make_prz_potential.py
"""
import itertools
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402
from oracle import oracle as O  # noqa: E402

W = __graft_entry__.load_package().workloads
OUT = os.path.join(ROOT, "tests", "golden", "prz")
RC = 11.0
HIDDEN = (16, 12)
ACTS = "p r l"


def rows():
    els = W.ABX3_ELEMENTS
    out = []
    for c in els:
        for e in els:
            for eta in (0.002, 0.05, 0.4):
                out.append((c, 2, e, 0, eta, 0.0, 0.0))
        for a, b in itertools.combinations_with_replacement(els, 2):
            for eta in (0.001, 0.013):
                for lam in (-1.0, 1.0):
                    for zeta in (1.0, 2.5, 6.3):
                        out.append((c, 3, a, b, eta, lam, zeta))
    return out


def write_input(d):
    S = W.SYMBOL
    L = ["# synthetic potential: softplus/ReLU layers, non-integer zeta",
         "number_of_elements 5",
         "elements " + " ".join(S[z] for z in W.ABX3_ELEMENTS),
         f"global_hidden_layers_short {len(HIDDEN)}",
         "global_nodes_short " + " ".join(str(h) for h in HIDDEN),
         "global_activation_short " + ACTS,
         "cutoff_type 2",
         "scale_symmetry_functions",
         "center_symmetry_functions"]
    for z in W.ABX3_ELEMENTS:
        L.append(f"atom_energy {S[z]} {-0.01 * z:.6f}")
    for c, t, a, b, eta, x, zeta in rows():
        if t == 2:
            L.append(f"symfunction_short {S[c]} 2 {S[a]} {eta:.6f} {x:.4f} {RC:.4f}")
        else:
            L.append(f"symfunction_short {S[c]} 3 {S[a]} {S[b]} {eta:.6f} {x:.1f} {zeta:.2f} {RC:.4f}")
    with open(os.path.join(d, "input.nn"), "w") as f:
        f.write("\n".join(L) + "\n")


def main():
    os.makedirs(OUT, exist_ok=True)
    write_input(OUT)
    nsf = len(rows()) // len(W.ABX3_ELEMENTS)
    W.write_abx3_weights(OUT, nsf=nsf, hidden=HIDDEN, seed=4321)
    W.write_scaling(OUT, [np.tile([0.0, 1.0, 0.0], (nsf, 1)) for _ in W.ABX3_ELEMENTS])
    m = O.Model(OUT)
    sample = [W.config_c2()] + W.config_c4(n_struct=64, seed=45)
    Gs = {z: [] for z in W.ABX3_ELEMENTS}
    for s in sample:
        G = m.symfunctions(s["Z"], s["pos"], s["lat"])
        for z in W.ABX3_ELEMENTS:
            Gs[z].append(G[s["Z"] == z, :nsf])
    stats = []
    for z in W.ABX3_ELEMENTS:
        g = np.concatenate(Gs[z])
        mn, mx, me = g.min(0), g.max(0), g.mean(0)
        width = np.maximum(mx - mn, np.maximum(0.5 * np.maximum(np.abs(mn), np.abs(mx)), 1e-6))
        stats.append(np.stack([mn, mn + width, me], 1))
    W.write_scaling(OUT, stats)
    m2 = O.Model(OUT)
    s = sample[0]
    G2 = m2.symfunctions(s["Z"], s["pos"], s["lat"])
    print("nsf", nsf, "scaled SF range:", G2[:, :nsf].min(), G2[:, :nsf].max())
    e = m2.eval(s["Z"], s["pos"], s["lat"])
    print("768-atom energy", e["energy"], "max |F|", np.abs(e["forces"]).max())


if __name__ == "__main__":
    main()
