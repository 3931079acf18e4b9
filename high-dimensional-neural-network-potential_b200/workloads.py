"""Seeded synthetic structures and the synthetic RuNNer potential.

No public dataset is involved: every structure is generated from a seed.

* ``abx3_cell()``: a 12-atom cubic ABX3-like cell (Pb, 3 I, a CH3-NH3 pair on
  the body diagonal), lattice constant 11.9 Bohr.
* ``supercell()``: repetition in the order of ``as_repeatUnitCell``
  (atomicStructure.f90:636-671): x outer, then y, then z, then atoms.
* ``config_c1`` ... ``config_c5``: the five benchmark workloads (methylammonium
  MD, 768-atom cell, 49,152-atom strained cell, 4096 mixed structures, 256
  served walkers).
* ``write_abx3_potential()``: RuNNer files (input.nn, weights.NNN.data) for the
  5-element, 280-SF/element potential with a 280-25-25-1 network; the
  ``scaling.data`` that goes with it is data (min/max/mean of each SF over the
  768-atom cell) and ships with the tests.

Positions are in Bohr; a structure is a dict with ``Z`` (int32[nat]),
``pos`` (float64[nat,3]), ``lat`` (float64[3,3], column c = lattice vector c)
or None for a molecule.
"""
from __future__ import annotations

import itertools
import os

import numpy as np

# Unit factors as used by the reference's MD example (constants.f90:10-12).
KBOLTZMANN = 3.166811965e-6  # Ha / K
AMU_TO_ME = 1822.888513874368
FS_TO_AU = 41.34137333519408

# Standard atomic weights of the elements the workloads use.
ATOMIC_MASS = {1: 1.008, 6: 12.011, 7: 14.007, 53: 126.904, 82: 207.2}
SYMBOL = {1: "H", 6: "C", 7: "N", 53: "I", 82: "Pb"}
Z_OF = {v: k for k, v in SYMBOL.items()}

ABX3_A = 11.9
ABX3_ELEMENTS = (1, 6, 7, 53, 82)


def abx3_cell(a: float = ABX3_A):
    """12 atoms: Pb at the origin, I at the three face/edge midpoints, C and N
    on the body diagonal at the centre -/+ 1.4 Bohr, three H on each of C and
    N at 1.95 Bohr from the axis and 0.7 Bohr outward along it."""
    u = np.ones(3) / np.sqrt(3.0)
    e1 = np.array([1.0, -1.0, 0.0]) / np.sqrt(2.0)
    e2 = np.cross(u, e1)
    c0 = np.full(3, a / 2)
    posC = c0 - 1.4 * u
    posN = c0 + 1.4 * u
    Z, P = [82, 53, 53, 53, 6, 7], [np.zeros(3), [a / 2, 0, 0], [0, a / 2, 0], [0, 0, a / 2], posC, posN]
    for base, sgn, phase in ((posC, -1.0, 0.0), (posN, 1.0, np.pi / 3)):
        for k in range(3):
            phi = phase + 2 * np.pi * k / 3
            P.append(base + sgn * 0.7 * u + 1.95 * (np.cos(phi) * e1 + np.sin(phi) * e2))
            Z.append(1)
    return {"Z": np.array(Z, np.int32), "pos": np.array(P, dtype=np.float64), "lat": np.eye(3) * a}


def supercell(s, n):
    nx, ny, nz = n
    lat = s["lat"]
    Z, P = [], []
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                shift = x * lat[:, 0] + y * lat[:, 1] + z * lat[:, 2]
                Z.append(s["Z"])
                P.append(s["pos"] + shift)
    L = lat.copy()
    L[:, 0] *= nx
    L[:, 1] *= ny
    L[:, 2] *= nz
    return {"Z": np.concatenate(Z).astype(np.int32), "pos": np.concatenate(P), "lat": L}


def strain(s, eps):
    """Affine strain h -> (I+eps) h applied to lattice and positions."""
    T = np.eye(3) + np.asarray(eps)
    return {"Z": s["Z"], "pos": s["pos"] @ T.T, "lat": T @ s["lat"]}


def read_xyz(path):
    """as_readXYZ (atomicStructure.f90:143-166): no unit conversion."""
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[0].split()[0])
    Z, P = [], []
    for l in lines[2 : 2 + n]:
        w = l.split()
        Z.append(Z_OF[w[0]])
        P.append([float(x) for x in w[1:4]])
    return {"Z": np.array(Z, np.int32), "pos": np.array(P), "lat": None}


# ------------------------------------------------------------------ configs
def config_c1(example_dir, seed=0, temperature=140.0):
    """Methylammonium (8 atoms, non-periodic) + masses and seeded momenta
    p0 = N(0,1) * sqrt(T kB m), centred (hdnnpExample.f90:39-49)."""
    s = read_xyz(os.path.join(example_dir, "input.xyz"))
    m = np.array([ATOMIC_MASS[int(z)] for z in s["Z"]]) * AMU_TO_ME
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((len(m), 3)) * np.sqrt(temperature * KBOLTZMANN * m)[:, None]
    p -= p.mean(axis=0)
    return s, m, p


def config_c2(seed=1, jitter=0.1):
    s = supercell(abx3_cell(), (4, 4, 4))
    rng = np.random.default_rng(seed)
    s["pos"] = s["pos"] + rng.normal(0.0, jitter, s["pos"].shape)
    return s


def config_c3(seed=2, n=16, max_strain=0.03):
    rng = np.random.default_rng(seed)
    eps = rng.uniform(-max_strain, max_strain, (3, 3))
    return strain(supercell(abx3_cell(), (n, n, n)), eps)


def maxwell_boltzmann(Z, temperature, seed):
    m = np.array([ATOMIC_MASS[int(z)] for z in Z]) * AMU_TO_ME
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((len(m), 3)) * np.sqrt(temperature * KBOLTZMANN * m)[:, None]
    p -= p.mean(axis=0)
    return m, p


def config_c4(n_struct=4096, seed=4, max_strain=0.05, jitter=0.15, max_rep=4):
    """Mixed sizes: nx, ny, nz ~ U{1..max_rep}, per-structure strain and jitter."""
    rng = np.random.default_rng(seed)
    cell = abx3_cell()
    out = []
    for _ in range(n_struct):
        n = tuple(int(v) for v in rng.integers(1, max_rep + 1, 3))
        eps = rng.uniform(-max_strain, max_strain, (3, 3))
        s = strain(supercell(cell, n), eps)
        s["pos"] = s["pos"] + rng.normal(0.0, jitter, s["pos"].shape)
        out.append(s)
    return out


def walker_shapes(lo=96, hi=3072):
    shapes = []
    for n in itertools.product(range(1, 9), repeat=3):
        nat = 12 * n[0] * n[1] * n[2]
        if lo <= nat <= hi:
            shapes.append(n)
    return shapes


def config_c5(n_walkers=256, seed=5, jitter=0.1):
    rng = np.random.default_rng(seed)
    shapes = walker_shapes()
    cell = abx3_cell()
    out = []
    for _ in range(n_walkers):
        n = shapes[int(rng.integers(0, len(shapes)))]
        s = supercell(cell, n)
        s["pos"] = s["pos"] + rng.normal(0.0, jitter, s["pos"].shape)
        out.append(s)
    return out


def concat(structs):
    """Batch CSR: atom offsets, flat Z/pos, lattices (identity for molecules)."""
    off = np.zeros(len(structs) + 1, np.int64)
    off[1:] = np.cumsum([len(s["Z"]) for s in structs])
    Z = np.concatenate([s["Z"] for s in structs]).astype(np.int32)
    pos = np.concatenate([s["pos"] for s in structs]).astype(np.float64)
    lat = np.stack([s["lat"] if s["lat"] is not None else np.eye(3) for s in structs])
    per = np.array([1 if s["lat"] is not None else 0 for s in structs], np.int32)
    return off, Z, pos, lat, per


# ------------------------------------------------------------------ potential
def abx3_symfunctions():
    """(centre, type, el1, el2, eta, rs_or_lambda, zeta) rows: per centre
    element 8 G2 per neighbour element (eta log-spaced 0.001..0.5, Rs=0) and
    16 G4 per unordered element pair (zeta 1,2,4,16 x lambda +-1 x eta
    0.001, 0.01): 40 + 240 = 280 per element."""
    els = ABX3_ELEMENTS
    etas2 = np.geomspace(0.001, 0.5, 8)
    rows = []
    for c in els:
        for e in els:
            for eta in etas2:
                rows.append((c, 2, e, 0, float(eta), 0.0, 0.0))
        for a, b in itertools.combinations_with_replacement(els, 2):
            for eta in (0.001, 0.01):
                for lam in (-1.0, 1.0):
                    for zeta in (1.0, 2.0, 4.0, 16.0):
                        rows.append((c, 3, a, b, eta, lam, zeta))
    return rows


def write_abx3_input(dirname, rc=12.0, hidden=(25, 25)):
    os.makedirs(dirname, exist_ok=True)
    L = [
        "# synthetic 5-element potential: 280 symmetry functions per element",
        "number_of_elements 5",
        "elements " + " ".join(SYMBOL[z] for z in ABX3_ELEMENTS),
        f"global_hidden_layers_short {len(hidden)}",
        "global_nodes_short " + " ".join(str(h) for h in hidden),
        "global_activation_short " + " ".join(["t"] * len(hidden) + ["l"]),
        "cutoff_type 2",
        "scale_symmetry_functions",
        "center_symmetry_functions",
    ]
    for c, t, a, b, eta, x, zeta in abx3_symfunctions():
        if t == 2:
            L.append(f"symfunction_short {SYMBOL[c]} 2 {SYMBOL[a]} {eta:.10f} {x:.4f} {rc:.4f}")
        else:
            L.append(f"symfunction_short {SYMBOL[c]} 3 {SYMBOL[a]} {SYMBOL[b]} {eta:.10f} {x:.1f} {zeta:.1f} {rc:.4f}")
    with open(os.path.join(dirname, "input.nn"), "w") as f:
        f.write("\n".join(L) + "\n")


def write_abx3_weights(dirname, nsf=280, hidden=(25, 25), seed=1234):
    """W ~ N(0, 1/fan_in), b ~ N(0, 1/fan_in), written in readWeights order
    (hdnnps.f90:318-327): per layer, for iin: for iout: W(iout, iin); then b."""
    rng = np.random.default_rng(seed)
    sizes = [nsf, *hidden, 1]
    for z in ABX3_ELEMENTS:
        vals = []
        for nin, nout in zip(sizes[:-1], sizes[1:]):
            W = rng.normal(0.0, 1.0 / np.sqrt(nin), (nout, nin))
            b = rng.normal(0.0, 1.0 / np.sqrt(nin), nout)
            vals.extend(W.T.reshape(-1))  # iin outer, iout inner
            vals.extend(b)
        with open(os.path.join(dirname, f"weights.{z:03d}.data"), "w") as f:
            f.write("\n".join(f"{v:.12e}" for v in vals) + "\n")


def write_scaling(dirname, stats, emin=-1.0, emax=1.0):
    """stats: list over elements (sorted by Z) of arrays (nsf, 3) = min, max, mean."""
    lines = []
    for ie, st in enumerate(stats):
        for isf, (mn, mx, me) in enumerate(st):
            lines.append(f"{ie + 1:4d} {isf + 1:4d} {mn:.12e} {mx:.12e} {me:.12e}")
    lines.append(f"{emin:.10f} {emax:.10f}")
    with open(os.path.join(dirname, "scaling.data"), "w") as f:
        f.write("\n".join(lines) + "\n")
