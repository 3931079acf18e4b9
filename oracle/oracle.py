"""ctypes wrapper of the FP64 CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module.  It restates the reference's prediction path
(hdnnps.f90:333 ``hdnnpEnergyAndForces`` and the routines it calls); see the
header of ``hdnnp_oracle.cpp`` for what pins it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liborc.so")
_lib = None
_native = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "hdnnp_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "lib/liborc.so"], check=True)
    return _LIB_PATH


def host_tag() -> str:
    """Short hash of this host's CPU model and instruction-set flags: the
    -march=native build is made for, and only loaded on, the CPU it names."""
    import hashlib
    import platform

    model = flags = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and not model:
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = line.split(":", 1)[1].strip()
                if model and flags:
                    break
    except OSError:
        pass
    return hashlib.sha1(f"{platform.machine()}|{model}|{flags}".encode()).hexdigest()[:12]


def build_native() -> str:
    """The same source built -O3 -march=native -fopenmp for this host (the
    timed CPU stand-in; the -O2 -ffp-contract=off build stays the checker)."""
    tag = host_tag()
    path = os.path.join(_HERE, "lib", f"liborc_native_{tag}.so")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(os.path.join(_HERE, "hdnnp_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE, "native", f"TAG={tag}"], check=True)
    return path


NATIVE_FLAGS = "g++ -O3 -march=native -fopenmp"
CHECKER_FLAGS = "g++ -O2 -ffp-contract=off -fopenmp"


def _bind(L):
    P, D, I = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.orc_last_error.restype = C.c_char_p
    L.orc_model_load.restype = P
    L.orc_model_load.argtypes = [C.c_char_p, C.c_int]
    L.orc_model_free.argtypes = [P]
    L.orc_model_info.argtypes = [P, I, I, I, D]
    L.orc_model_sfs.argtypes = [P, C.c_int, D]
    L.orc_model_net.argtypes = [P, C.c_int, I, I, C.c_char_p, D]
    L.orc_model_flags.argtypes = [P, I, I, D]
    L.orc_neighbours.argtypes = [P, C.c_int, I, D, C.c_int, D, C.c_int, C.c_int, I, I, D]
    L.orc_symfunctions.argtypes = [P, C.c_int, I, D, C.c_int, D, C.c_int, C.c_int, D, C.c_int, D]
    L.orc_eval.argtypes = [P, C.c_int, I, D, C.c_int, D, D, D, D, D, D, C.c_int, C.c_int, C.c_int]
    L.orc_dEdLat_to_stress.argtypes = [D, D, D]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_max_threads.restype = C.c_int
    return L


def lib(native: bool = False):
    """The checker build (default), or with native=True the -O3
    -march=native build of the same source for timing."""
    global _lib, _native
    if native:
        if _native is None:
            _native = _bind(C.CDLL(build_native()))
        return _native
    if _lib is None:
        build()
        _lib = _bind(C.CDLL(_LIB_PATH))
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class OracleError(RuntimeError):
    pass


class Model:
    """parseRuNNerInput (hdnnps.f90:34).  ``path`` is a directory.
    native=True runs the -O3 -march=native build (timing only)."""

    def __init__(self, path: str, cap_sfs: int = 0, native: bool = False):
        p = path if path.endswith("/") else path + "/"
        self._L = lib(native)
        self._h = self._L.orc_model_load(p.encode(), int(cap_sfs))
        if not self._h:
            raise OracleError(self._L.orc_last_error().decode())
        nel = C.c_int()
        zs = np.zeros(128, np.int32)
        nsf = np.zeros(128, np.int32)
        rc = C.c_double()
        self._L.orc_model_info(self._h, C.byref(nel), _i(zs), _i(nsf), C.byref(rc))
        self.elements = [int(z) for z in zs[: nel.value]]
        self.nsf = {int(z): int(n) for z, n in zip(zs[: nel.value], nsf[: nel.value])}
        self.max_rc = rc.value
        self.max_nsf = max(self.nsf.values())

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.orc_model_free(self._h)
            self._h = None

    def sfs(self, z: int) -> np.ndarray:
        out = np.zeros((self.nsf[z], 11))
        self._L.orc_model_sfs(self._h, int(z), _d(out))
        return out

    def net(self, z: int):
        nl = C.c_int()
        dims = np.zeros(64, np.int32)
        acts = C.create_string_buffer(32)
        self._L.orc_model_net(self._h, int(z), C.byref(nl), _i(dims), acts, None)
        n = nl.value
        shapes = [(int(dims[2 * l]), int(dims[2 * l + 1])) for l in range(n)]
        total = sum(i * o + o for i, o in shapes)
        w = np.zeros(total)
        self._L.orc_model_net(self._h, int(z), C.byref(nl), _i(dims), acts, _d(w))
        layers, off = [], 0
        for (nin, nout), a in zip(shapes, acts.raw[:n].decode()):
            W = w[off : off + nin * nout].reshape(nin, nout).T.copy()  # (nout, nin)
            off += nin * nout
            b = w[off : off + nout].copy()
            off += nout
            layers.append((W, b, a))
        return layers

    def flags(self):
        s, c = C.c_int(), C.c_int()
        ae = np.zeros(119)
        self._L.orc_model_flags(self._h, C.byref(s), C.byref(c), _d(ae))
        return bool(s.value), bool(c.value), ae

    # ------------------------------------------------------------------ stages
    def neighbours(self, Z, pos, lat=None, brute=False, cap=256):
        Z, pos, lat, per = _prep(Z, pos, lat)
        n = len(Z)
        counts = np.zeros(n, np.int32)
        idx = np.zeros(n * cap, np.int32)
        npos = np.zeros(n * cap * 3)
        mx = self._L.orc_neighbours(self._h, n, _i(Z), _d(pos), per, _d(lat), 1 if brute else 0, cap, _i(counts), _i(idx), _d(npos))
        if mx > cap:
            return self.neighbours(Z, pos, lat if per else None, brute, cap=mx)
        return counts, idx.reshape(n, cap), npos.reshape(n, cap, 3)

    def symfunctions(self, Z, pos, lat=None, separate=False, with_grad=False, cap=64):
        Z, pos, lat, per = _prep(Z, pos, lat)
        n = len(Z)
        G = np.zeros((n, self.max_nsf))
        dG = np.zeros((n, self.max_nsf, cap, 3)) if with_grad else None
        r = self._L.orc_symfunctions(self._h, n, _i(Z), _d(pos), per, _d(lat), int(separate), self.max_nsf, _d(G), cap, _d(dG))
        if r != 0:
            raise OracleError(self._L.orc_last_error().decode())
        return (G, dG) if with_grad else G

    def eval(self, Z, pos, lat=None, stress=True, brute=False, separate=False, per_atom=False):
        """Energy, forces (nat,3), dEdLat (3,3 Fortran layout: [row][col]) or None."""
        Z, pos, lat, per = _prep(Z, pos, lat)
        n = len(Z)
        E = C.c_double()
        F = np.zeros(3 * n)
        dl = np.zeros(9) if (per and stress) else None
        atE = np.zeros(n) if per_atom else None
        dEdG = np.zeros((n, self.max_nsf)) if per_atom else None
        r = self._L.orc_eval(self._h, n, _i(Z), _d(pos), per, _d(lat), C.byref(E), _d(F), _d(dl), _d(atE), _d(dEdG), self.max_nsf, int(brute), int(separate))
        if r != 0:
            raise OracleError(self._L.orc_last_error().decode())
        out = {"energy": E.value, "forces": F.reshape(n, 3),
               "dEdLat": dl.reshape(3, 3, order="F") if dl is not None else None}
        if per_atom:
            out["atom_energies"] = atE
            out["dEdG"] = dEdG
        return out


def dEdLat_to_stress(lat: np.ndarray, dEdLat: np.ndarray) -> np.ndarray:
    """dEdLat2Stress (atomicStructure.f90:679); lat[:, c] = lattice vector c."""
    latf = np.asfortranarray(lat, dtype=np.float64).ravel(order="F").copy()
    dl = np.asarray(dEdLat, dtype=np.float64).ravel(order="F").copy()
    out = np.zeros(9)
    lib().orc_dEdLat_to_stress(_d(latf), _d(dl), _d(out))
    return out.reshape(3, 3, order="F")


def _prep(Z, pos, lat):
    Z = np.ascontiguousarray(Z, dtype=np.int32)
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    if lat is None:
        return Z, pos, np.zeros(9), 0
    # lat[:, c] is lattice vector c -> Fortran column-major flat array
    latf = np.asarray(lat, dtype=np.float64).ravel(order="F").copy()
    return Z, pos, latf, 1
