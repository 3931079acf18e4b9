"""Writes tests/golden/oracle_fixtures.json: oracle outputs for the example
methylammonium molecule and a strained, jittered 12-atom ABX3 cell (seed 7).
These pin the oracle against regressions and give the GPU parity tests a
committed target.  Run from the repository root."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import __graft_entry__  # noqa: E402
from oracle import oracle as O  # noqa: E402
from test_oracle import small_cell  # noqa: E402

W = __graft_entry__.load_package().workloads
G = os.path.join(ROOT, "tests", "golden")


def main():
    O.set_threads(1)
    ex = O.Model(os.path.join(G, "example"))
    ab = O.Model(os.path.join(G, "abx3"))
    s = W.read_xyz(os.path.join(G, "example", "input.xyz"))
    r1 = ex.eval(s["Z"], s["pos"], per_atom=True)
    c = small_cell(W)
    r2 = ab.eval(c["Z"], c["pos"], c["lat"], per_atom=True)
    out = {
        "c1": {"energy": r1["energy"], "forces": r1["forces"].tolist(), "atom_energies": r1["atom_energies"].tolist()},
        "cell": {"Z": c["Z"].tolist(), "pos": c["pos"].tolist(), "lat": c["lat"].tolist(),
                 "energy": r2["energy"], "forces": r2["forces"].tolist(), "dEdLat": r2["dEdLat"].tolist(),
                 "atom_energies": r2["atom_energies"].tolist()},
    }
    with open(os.path.join(G, "oracle_fixtures.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
