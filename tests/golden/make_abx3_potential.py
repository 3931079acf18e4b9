"""Generates the synthetic ABX3 potential used by the 768-atom, 49k-atom,
batched and served workloads (tests/golden/abx3/).

input.nn and weights.NNN.data come from hdnnp_b200.workloads (seed 1234).
scaling.data holds min/max/mean of every symmetry function over a
"training" sample: the 768-atom jittered supercell (seed 1) and 256
structures drawn like the batched workload (seed 44, not a benchmark seed),
computed with the FP64 oracle on unscaled SFs.  Each range is floored at half
of the SF's largest magnitude (and at 1e-6): several angular SFs of this
lattice are tiny and nearly constant (Pb-Pb pairs sit at 11.9 Bohr, just
inside rc = 12), and an unfloored range of ~1e-12 would turn rounding noise
into O(1) network inputs.
Run from the repository root:  python tests/golden/make_abx3_potential.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402
from oracle import oracle as O  # noqa: E402

W = __graft_entry__.load_package().workloads
OUT = os.path.join(ROOT, "tests", "golden", "abx3")


def main():
    W.write_abx3_input(OUT)
    W.write_abx3_weights(OUT)
    # identity scaling first: centre by 0, divide by 1
    idstats = [np.tile([0.0, 1.0, 0.0], (280, 1)) for _ in W.ABX3_ELEMENTS]
    W.write_scaling(OUT, idstats)
    m = O.Model(OUT)
    sample = [W.config_c2()] + W.config_c4(n_struct=256, seed=44)
    Gs = {z: [] for z in W.ABX3_ELEMENTS}
    for s in sample:
        G = m.symfunctions(s["Z"], s["pos"], s["lat"])
        for z in W.ABX3_ELEMENTS:
            Gs[z].append(G[s["Z"] == z, :280])
    stats = []
    for z in W.ABX3_ELEMENTS:
        g = np.concatenate(Gs[z])
        mn, mx, me = g.min(0), g.max(0), g.mean(0)
        width = np.maximum(mx - mn, np.maximum(0.5 * np.maximum(np.abs(mn), np.abs(mx)), 1e-6))
        stats.append(np.stack([mn, mn + width, me], 1))
    W.write_scaling(OUT, stats)
    m2 = O.Model(OUT)
    G2 = m2.symfunctions(s["Z"], s["pos"], s["lat"])
    print("scaled SF range:", G2[:, :280].min(), G2[:, :280].max())


if __name__ == "__main__":
    main()
