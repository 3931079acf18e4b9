"""Structure files in the formats the reference reads and writes
(src/atoms/atomicStructure.f90), feeding batches of the engine.

A structure is a dict with ``Z`` (int32[nat]), ``pos`` (float64[nat, 3],
Bohr) and ``lat`` (float64[3, 3], column c = lattice vector c, Bohr) or None
for a molecule; ``read_data`` adds ``energy``, ``charge``, ``q`` and ``forces``.

=================  ==========================  =====================================
format             reference                   here
=================  ==========================  =====================================
xyz                as_readXYZ / as_writeXYZ    read_xyz / write_xyz
                   (:143, :224)                (no unit conversion, as the reference)
FHI-aims           as_readFhiaims (:168)       read_fhiaims / write_fhiaims (Angstrom)
v_sim ascii        as_readAscii /              read_ascii / write_ascii
                   as_writeAscii (:245, :288)  (optional 'angstroem'; lattice aligned)
RuNNer data        as_readData /               read_data / write_data
                   as_writeDataToUnit          (begin/lattice/atom/energy/charge/end)
                   (:354, :329)
POSCAR             as_readPOSCAR /             read_poscar / write_poscar
                   as_writePOSCAR (:427, :481) (Direct coordinates, Angstrom)
=================  ==========================  =====================================

Differences from the reference: the writers keep full precision (the
reference's xyz writer keeps 6 significant digits, ``'(A2,3E15.6)'``), and
errors raise ``ValueError`` instead of stopping.  Like the reference, the
POSCAR scale line is read and ignored, and an unknown element symbol maps to
Z = -1 (the engine rejects it when evaluating).
"""
from __future__ import annotations

import numpy as np

# constants.f90:7
ANG2BOHR = 1.8897259886

SYMBOLS = (
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca",
    "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",
    "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce",
    "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir",
    "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu", "Am", "Cm",
    "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds", "Rg", "Cn", "Nh", "Fl", "Mc",
    "Lv", "Ts", "Og")
_Z = {s: i + 1 for i, s in enumerate(SYMBOLS)}


def sym_to_z(sym: str) -> int:
    """elemSymToNum (constants.f90:95): exact symbol match, -1 if unknown."""
    return _Z.get(sym.strip(), -1)


def z_to_sym(z: int) -> str:
    """elemNumToSym (constants.f90:84): 'XX' beyond 118."""
    return SYMBOLS[z - 1] if 1 <= z <= 118 else "XX"


def _fmt(x: float) -> str:
    return repr(float(x))  # shortest representation that reads back bitwise


def _struct(Z, pos, lat):
    return {"Z": np.asarray(Z, np.int32), "pos": np.asarray(pos, float).reshape(-1, 3),
            "lat": None if lat is None else np.asarray(lat, float).reshape(3, 3)}


# ----------------------------------------------------------------------- xyz
def read_xyz(path):
    """as_readXYZ: nat, a comment line, then 'El x y z'; a molecule."""
    with open(path) as f:
        lines = f.read().splitlines()
    nat = int(lines[0].split()[0])
    Z, pos = [], []
    for ln in lines[2:2 + nat]:
        t = ln.split()
        Z.append(sym_to_z(t[0]))
        pos.append([float(v) for v in t[1:4]])
    if len(Z) != nat:
        raise ValueError(f"{path}: {nat} atoms announced, {len(Z)} found")
    return _struct(Z, pos, None)


def write_xyz(path, s, comment=""):
    with open(path, "w") as f:
        f.write(f"{len(s['Z'])}\n{comment}\n")
        for z, p in zip(s["Z"], s["pos"]):
            f.write(f"{z_to_sym(int(z))} {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}\n")


# ----------------------------------------------------------------------- FHI-aims
def read_fhiaims(path):
    """as_readFhiaims: 'atom x y z El' and up to three 'lattice_vector x y z'
    lines, in Angstrom; periodic when a lattice vector is given."""
    Z, pos, lat = [], [], []
    with open(path) as f:
        for ln in f:
            if ln.startswith("atom"):
                t = ln.split()
                pos.append([float(v) for v in t[1:4]])
                Z.append(sym_to_z(t[4]))
            elif ln.startswith("lattice_vector"):
                if len(lat) == 3:
                    raise ValueError(f"{path}: more than 3 lattice vectors")
                lat.append([float(v) for v in ln.split()[1:4]])
    L = None
    if lat:
        L = np.zeros((3, 3))
        for c, v in enumerate(lat):
            L[:, c] = v
        L = L * ANG2BOHR
    return _struct(Z, np.asarray(pos, float) * ANG2BOHR, L)


def write_fhiaims(path, s):
    with open(path, "w") as f:
        if s["lat"] is not None:
            for c in range(3):
                v = s["lat"][:, c] / ANG2BOHR
                f.write(f"lattice_vector {_fmt(v[0])} {_fmt(v[1])} {_fmt(v[2])}\n")
        for z, p in zip(s["Z"], s["pos"] / ANG2BOHR):
            f.write(f"atom {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])} {z_to_sym(int(z))}\n")


# ----------------------------------------------------------------------- v_sim ascii
def read_ascii(path, is_angstrom=False):
    """as_readAscii: 'nat [angstroem]', then dxx dyx dyy and dzx dzy dzz (the
    lattice in lower-triangular form), then 'x y z El'; always periodic."""
    with open(path) as f:
        lines = f.read().splitlines()
    head = lines[0].split()
    nat = int(head[0])
    angs = is_angstrom or (len(head) > 1 and head[1][:9] == "angstroem")
    a = [float(v) for v in lines[1].split()[:3]]
    b = [float(v) for v in lines[2].split()[:3]]
    L = np.zeros((3, 3))
    L[0, 0] = a[0]
    L[0, 1], L[1, 1] = a[1], a[2]
    L[:, 2] = b
    Z, pos = [], []
    for ln in lines[3:3 + nat]:
        t = ln.split()
        pos.append([float(v) for v in t[:3]])
        Z.append(sym_to_z(t[3]))
    pos = np.asarray(pos, float)
    if angs:
        pos, L = pos * ANG2BOHR, L * ANG2BOHR
    return _struct(Z, pos, L)


def align_lattice_with_axes(lat, pos):
    """alignLatticeWithAxes (pointsets.f90:148): lat = Q R (Householder QR);
    the lattice becomes R (vector 1 along x, vector 2 in the xy plane) and the
    positions are rotated by Q^T; Q and R change sign when the trace of Q is
    negative."""
    Q, R = np.linalg.qr(np.asarray(lat, float))
    if Q[0, 0] + Q[1, 1] + Q[2, 2] < 0.0:
        Q, R = -Q, -R
    return R, np.asarray(pos, float) @ Q  # rows: Q^T p


def write_ascii(path, s, to_angstrom=False):
    if s["lat"] is None:
        raise ValueError("the ascii format needs a periodic structure")
    lat, pos = s["lat"], s["pos"]
    if to_angstrom:
        lat, pos = lat / ANG2BOHR, pos / ANG2BOHR
    lat, pos = align_lattice_with_axes(lat, pos)
    with open(path, "w") as f:
        f.write(f"{len(s['Z'])}{' angstroem' if to_angstrom else ''}\n")
        f.write(f"{_fmt(lat[0, 0])} {_fmt(lat[0, 1])} {_fmt(lat[1, 1])}\n")
        f.write(f"{_fmt(lat[0, 2])} {_fmt(lat[1, 2])} {_fmt(lat[2, 2])}\n")
        for z, p in zip(s["Z"], pos):
            f.write(f"{_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])} {z_to_sym(int(z))}\n")


# ----------------------------------------------------------------------- RuNNer data
def read_data(path):
    """as_readData: blocks 'begin' ... 'end' with 'lattice x y z' (three make a
    periodic structure), 'atom x y z El q e fx fy fz', 'energy E', 'charge Q'."""
    out, cur = [], None
    with open(path) as f:
        for raw in f:
            ln = raw.strip()
            if ln.startswith("begin"):
                cur = {"lat": [], "pos": [], "Z": [], "q": [], "forces": [], "energy": 0.0, "charge": 0.0}
            elif cur is None:
                continue
            elif ln.startswith("lattice"):
                cur["lat"].append([float(v) for v in ln.split()[1:4]])
            elif ln.startswith("atom"):
                t = ln.split()
                cur["pos"].append([float(v) for v in t[1:4]])
                cur["Z"].append(sym_to_z(t[4]))
                cur["q"].append(float(t[5]))
                cur["forces"].append([float(v) for v in t[7:10]])
            elif ln.startswith("energy"):
                cur["energy"] = float(ln.split()[1])
            elif ln.startswith("charge"):
                cur["charge"] = float(ln.split()[1])
            elif ln.startswith("end"):
                L = None
                if len(cur["lat"]) == 3:
                    L = np.asarray(cur["lat"], float).T  # column c = lattice vector c
                s = _struct(cur["Z"], cur["pos"], L)
                s.update(energy=cur["energy"], charge=cur["charge"], q=np.asarray(cur["q"], float),
                         forces=np.asarray(cur["forces"], float).reshape(-1, 3))
                out.append(s)
                cur = None
    return out


def write_data(path, structs, energies=None, forces=None, charges=None):
    """as_writeDataToUnit for each structure (append mode is the caller's)."""
    with open(path, "w") as f:
        for k, s in enumerate(structs):
            n = len(s["Z"])
            E = energies[k] if energies is not None else s.get("energy", 0.0)
            F = forces[k] if forces is not None else s.get("forces", np.zeros((n, 3)))
            q = charges[k] if charges is not None else s.get("q", np.zeros(n))
            f.write("begin\n")
            if s["lat"] is not None:
                for c in range(3):
                    v = s["lat"][:, c]
                    f.write(f"lattice {_fmt(v[0])} {_fmt(v[1])} {_fmt(v[2])}\n")
            for z, p, qi, fi in zip(s["Z"], s["pos"], q, np.asarray(F).reshape(-1, 3)):
                f.write(f"atom {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])} {z_to_sym(int(z))} {_fmt(qi)} 0.0 "
                        f"{_fmt(fi[0])} {_fmt(fi[1])} {_fmt(fi[2])}\n")
            f.write(f"energy {_fmt(E)}\ncharge {int(round(float(np.sum(q))))}\nend\n")


# ----------------------------------------------------------------------- POSCAR
def read_poscar(path):
    """as_readPOSCAR: comment, scale (read, not applied, as in the reference),
    three lattice vectors (Angstrom), element symbols, counts, 'Direct', then
    fractional coordinates."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    L = np.zeros((3, 3))
    for c in range(3):
        L[:, c] = [float(v) for v in lines[2 + c].split()[:3]]
    L *= ANG2BOHR
    els = lines[5].split()
    counts = [int(v) for v in lines[6].split()]
    if lines[7].strip().lower() != "direct":
        raise ValueError(f"{path}: POSCAR without Direct coordinates is not supported")
    Z = [sym_to_z(e) for e, n in zip(els, counts) for _ in range(n)]
    frac = np.asarray([[float(v) for v in ln.split()[:3]] for ln in lines[8:8 + len(Z)]], float)
    return _struct(Z, frac @ L.T, L)


def write_poscar(path, s):
    """as_writePOSCAR: atoms grouped by distinct element in order of first
    appearance, fractional coordinates."""
    if s["lat"] is None:
        raise ValueError("POSCAR needs a periodic structure")
    Z = np.asarray(s["Z"])
    els = list(dict.fromkeys(int(z) for z in Z))
    frac = np.linalg.solve(s["lat"], s["pos"].T).T
    with open(path, "w") as f:
        f.write("\n1.0\n")
        for c in range(3):
            v = s["lat"][:, c] / ANG2BOHR
            f.write(f"{_fmt(v[0])} {_fmt(v[1])} {_fmt(v[2])}\n")
        f.write(" ".join(z_to_sym(e) for e in els) + "\n")
        f.write(" ".join(str(int(np.sum(Z == e))) for e in els) + "\nDIRECT\n")
        for e in els:
            for p in frac[Z == e]:
                f.write(f"{_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}\n")


READERS = {"xyz": read_xyz, "fhiaims": read_fhiaims, "ascii": read_ascii, "poscar": read_poscar}


def read_batch(paths, fmt):
    """Structures from many files (data files may hold several each), in order."""
    out = []
    for p in paths:
        out.extend(read_data(p) if fmt == "data" else [READERS[fmt](p)])
    return out
