"""Python mirror of the reference's potential API over the C ABI.

``Hdnnp`` stands for ``type(hdnnp)`` plus its routines in
src/potentials/hdnnps.f90:

=============================  ==============================================
reference (Fortran)            here
=============================  ==============================================
parseRuNNerInput(h, path)      ``Hdnnp.from_runner(path)``       (:34)
hdnnpEnergyAndForces(h, ats,   ``h.energy_and_forces(ats, dEdLat=True)``
  energy, force, dEdLat)        -> (energy, force(nat,3), dEdLat(3,3)) (:333)
type atStruct                  ``AtStruct``         (atomicStructure.f90:17)
dEdLat2Stress(lat, dEdLat, s)  ``dEdLat_to_stress`` (atomicStructure.f90:679)
globalHdnnpEnergyAndForces(    ``h.committee_energy_and_forces(members, ats)``
  ats, energy, forces,          -> (energy, forces, dEdLat, std)
  dEdLat, std)                  (globalHdnnps.f90:31)
hdnnpCalcNeighborLists(h, ats, ``h.calc_neighbor_lists(ats)``        (:373)
  neiLists)
hdnnpCalcSymfunctions(h, ats,  ``h.calc_symfunctions()`` -> G        (:390)
  neiLists, sfs)
hdnnpCalcNNs(h, ats, neiLists, ``h.calc_nns(nn=None, dEdLat=False)`` (:487)
  sfs, energy, force, dEdLat)
handle%sfLists / nnList /      ``h.symfunctions(z)``, ``h.network(z)``,
  scalesf / centersf / ...      ``h.flags()``                      (:13-21)
=============================  ==============================================

Errors that make the reference ``stop`` raise ``HdnnpError`` here.  Arrays
follow the reference layout: ``ats[:, i]`` would be the Fortran column of atom
i; in numpy we take ``pos`` of shape (nat, 3) (same memory order as the
Fortran (3, nat) array) and ``lat`` of shape (3, 3) with ``lat[:, c]`` =
lattice vector c.

The compute path is ``lib/libhdnnp_b200.so``; if it is missing or cannot be
loaded every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libhdnnp_b200.so")

HDNNP_PREC_FP64 = 0
HDNNP_PREC_MIXED = 1

_lib = None


class HdnnpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hdnnp error {code}: {msg}")
        self.code = code


def lib():
    """Loads libhdnnp_b200.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HdnnpError(-1, f"{LIB_PATH} is missing: build it with build.py (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    P, D, I, I64 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    L.hdnnp_last_error.restype = C.c_char_p
    L.hdnnp_model_load_runner.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    L.hdnnp_model_info.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), D]
    L.hdnnp_model_free.argtypes = [P]
    L.hdnnp_model_free.restype = None
    L.hdnnp_ctx_create.argtypes = [P, C.POINTER(C.c_void_p)]
    L.hdnnp_ctx_free.argtypes = [P]
    L.hdnnp_ctx_free.restype = None
    L.hdnnp_ctx_set_precision.argtypes = [P, C.c_int]
    L.hdnnp_ctx_set_option.argtypes = [P, C.c_char_p, C.c_int]
    L.hdnnp_energy_and_forces.argtypes = [P, C.c_int, I, D, C.c_int, D, D, D, D]
    L.hdnnp_eval_batch.argtypes = [P, C.c_int, I64, I, D, I, D, D, D, D]
    L.hdnnp_eval_batch_device.argtypes = [P, C.c_int, I64, P, P, P, I, D, P, P, P, P]
    L.hdnnp_dEdLat_to_stress.argtypes = [D, D, D]
    L.hdnnp_debug_fetch.argtypes = [P, C.c_char_p, P, C.c_size_t]
    L.hdnnp_last_launch_count.argtypes = [P, C.POINTER(C.c_int)]
    L.hdnnp_debug_math.argtypes = [C.c_int, C.c_int, D, D]
    L.hdnnp_ctx_set_profiling.argtypes = [P, C.c_int]
    L.hdnnp_profile_read.argtypes = [P, D, I64, C.c_int]
    L.hdnnp_committee_energy_and_forces.argtypes = [P, P, C.c_int, C.c_int, I, D, C.c_int, D, D, D, D, D]
    L.hdnnp_committee_eval_batch.argtypes = [P, P, C.c_int, C.c_int, I64, I, D, I, D, D, D, D, D]
    L.hdnnp_calc_neighbor_lists.argtypes = [P, C.c_int, I, D, C.c_int, D, C.POINTER(C.c_int)]
    L.hdnnp_calc_symfunctions.argtypes = [P, D]
    L.hdnnp_neighbor_lists_fetch.argtypes = [P, I, I, D]
    L.hdnnp_calc_nns.argtypes = [P, P, D, D, D]
    L.hdnnp_model_flags.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), D, D, D]
    L.hdnnp_model_symfunctions.argtypes = [P, C.c_int, C.POINTER(C.c_int), D]
    L.hdnnp_model_network.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, D]
    L.hdnnp_server_create.argtypes = [P, P, C.POINTER(C.c_void_p)]
    L.hdnnp_server_destroy.argtypes = [P]
    L.hdnnp_server_destroy.restype = None
    L.hdnnp_server_add_walker.argtypes = [P, C.c_int, I, D, C.c_int, D, D, D, C.POINTER(C.c_int)]
    L.hdnnp_server_remove_walker.argtypes = [P, C.c_int]
    L.hdnnp_server_submit.argtypes = [P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64,
                                      C.POINTER(C.c_uint64)]
    L.hdnnp_server_wait.argtypes = [P, C.c_uint64, C.c_int, D, D, D, D]
    L.hdnnp_server_next_done.argtypes = [P, C.c_int, C.POINTER(C.c_uint64)]
    L.hdnnp_server_read_walker.argtypes = [P, C.c_int, D, D]
    L.hdnnp_server_stats.argtypes = [P, D, D, D, D, C.POINTER(C.c_size_t), C.c_int]
    L.hdnnp_server_list_stats.argtypes = [P, I64, I64]
    _lib = L
    return L


def _check(code: int):
    if code != 0:
        raise HdnnpError(code, lib().hdnnp_last_error().decode())


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


@dataclass
class AtStruct:
    """type atStruct (atomicStructure.f90:17-28), prediction fields only."""

    el: np.ndarray                      # atomic numbers (nat,)
    ats: np.ndarray                     # positions (nat, 3), Bohr
    lat: Optional[np.ndarray] = None    # (3, 3), lat[:, c] = lattice vector c
    periodic: bool = field(default=False)

    def __post_init__(self):
        self.el = np.ascontiguousarray(self.el, dtype=np.int32)
        self.ats = np.ascontiguousarray(self.ats, dtype=np.float64).reshape(-1, 3)
        if self.lat is not None:
            self.lat = np.asarray(self.lat, dtype=np.float64).reshape(3, 3)
            self.periodic = True if self.periodic is False else self.periodic

    @property
    def nat(self) -> int:
        return len(self.el)


def _lat_flat(lat):
    if lat is None:
        return np.eye(3).ravel(order="F").copy()
    return np.asarray(lat, dtype=np.float64).ravel(order="F").copy()


class Hdnnp:
    """A potential on one GPU with one evaluation context."""

    def __init__(self, model_handle, device: int):
        self._m = model_handle
        self.device = device
        ctx = C.c_void_p()
        _check(lib().hdnnp_ctx_create(self._m, C.byref(ctx)))
        self._c = ctx
        n = C.c_int()
        zs = (C.c_int * 128)()
        ns = (C.c_int * 128)()
        rc = C.c_double()
        _check(lib().hdnnp_model_info(self._m, C.byref(n), zs, ns, C.byref(rc)))
        self.elements = [zs[i] for i in range(n.value)]
        self.nsf = {zs[i]: ns[i] for i in range(n.value)}
        self.max_rc = rc.value
        self.precision = HDNNP_PREC_FP64

    @classmethod
    def from_runner(cls, path: str, device: int = 0) -> "Hdnnp":
        """parseRuNNerInput (hdnnps.f90:34)."""
        h = C.c_void_p()
        _check(lib().hdnnp_model_load_runner(os.fsencode(path), int(device), C.byref(h)))
        return cls(h, device)

    def close(self):
        if getattr(self, "_c", None):
            lib().hdnnp_ctx_free(self._c)
            self._c = None
        if getattr(self, "_m", None):
            lib().hdnnp_model_free(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, name: str, value: int):
        _check(lib().hdnnp_ctx_set_option(self._c, name.encode(), int(value)))

    def set_precision(self, mode: int):
        _check(lib().hdnnp_ctx_set_precision(self._c, int(mode)))
        self.precision = mode

    # ------------------------------------------------------------------ evaluation
    def energy_and_forces(self, ats: AtStruct, dEdLat: bool = False):
        """hdnnpEnergyAndForces (hdnnps.f90:333): energy, forces (nat,3),
        and dE/dh (3,3) when ``dEdLat`` (periodic structures only)."""
        n = ats.nat
        E = C.c_double()
        F = np.zeros((n, 3))
        dl = np.zeros(9) if dEdLat else None
        _check(lib().hdnnp_energy_and_forces(
            self._c, n, _ip(ats.el), _dp(ats.ats), 1 if ats.periodic else 0,
            _dp(_lat_flat(ats.lat)), C.byref(E), _dp(F), _dp(dl)))
        return E.value, F, (dl.reshape(3, 3, order="F") if dl is not None else None)

    def eval_batch(self, structs: Sequence[dict], dEdLat: bool = True):
        """Independent structures in one batch (dicts with Z, pos, lat)."""
        off = np.zeros(len(structs) + 1, np.int64)
        off[1:] = np.cumsum([len(s["Z"]) for s in structs])
        Z = np.ascontiguousarray(np.concatenate([s["Z"] for s in structs]), dtype=np.int32)
        pos = np.ascontiguousarray(np.concatenate([s["pos"] for s in structs]), dtype=np.float64)
        lat = np.concatenate([_lat_flat(s["lat"]) for s in structs])
        per = np.array([0 if s["lat"] is None else 1 for s in structs], np.int32)
        return self.eval_batch_arrays(off, Z, pos, per, lat, dEdLat)

    # ------------------------------------------------------------------ stages
    def calc_neighbor_lists(self, ats: AtStruct) -> int:
        """hdnnpCalcNeighborLists (hdnnps.f90:373): the lists stay on the
        device in this potential's context; returns the neighbour entries."""
        n = C.c_int()
        _check(lib().hdnnp_calc_neighbor_lists(self._c, ats.nat, _ip(ats.el), _dp(ats.ats), 1 if ats.periodic else 0,
                                               _dp(_lat_flat(ats.lat)), C.byref(n)))
        self._stage_nat = ats.nat
        return n.value

    def neighbor_lists(self):
        """The lists of the last calc_neighbor_lists as the reference's
        neighborList (neighborLists.f90:10-16): per atom (iNeis, neis(nNei,
        3)), entry 0 the atom itself, 0-based indices."""
        n = np.zeros(self._stage_nat, np.int32)
        _check(lib().hdnnp_neighbor_lists_fetch(self._c, _ip(n), None, None))
        tot = int(n.sum())
        idx = np.zeros(tot, np.int32)
        pos = np.zeros((tot, 3))
        _check(lib().hdnnp_neighbor_lists_fetch(self._c, _ip(n), _ip(idx), _dp(pos)))
        off = np.concatenate([[0], np.cumsum(n)])
        return [(idx[off[i]:off[i + 1]], pos[off[i]:off[i + 1]]) for i in range(len(n))]

    def calc_symfunctions(self, fetch: bool = True):
        """hdnnpCalcSymfunctions (hdnnps.f90:390): scaled G of the structure
        of the last calc_neighbor_lists, (nat, nsf_max) when ``fetch``."""
        G = np.zeros((self._stage_nat, max(self.nsf.values()))) if fetch else None
        _check(lib().hdnnp_calc_symfunctions(self._c, _dp(G)))
        return G

    def calc_nns(self, nn: Optional["Hdnnp"] = None, dEdLat: bool = False):
        """hdnnpCalcNNs (hdnnps.f90:487): the networks of ``nn`` (default:
        this potential) on this context's symmetry functions; energy, forces
        (nat, 3) and dE/dh (3, 3) or None."""
        E = C.c_double()
        F = np.zeros((self._stage_nat, 3))
        dl = np.zeros(9) if dEdLat else None
        _check(lib().hdnnp_calc_nns(self._c, None if nn is None else nn._m, C.byref(E), _dp(F), _dp(dl)))
        return E.value, F, (dl.reshape(3, 3, order="F") if dl is not None else None)

    # ------------------------------------------------------------------ type(hdnnp) components
    def flags(self):
        """scalesf, centersf, emin, emax and atomenergies(118) (hdnnps.f90:13-21)."""
        sc, ce = C.c_int(), C.c_int()
        emin, emax = C.c_double(), C.c_double()
        ae = np.zeros(118)
        _check(lib().hdnnp_model_flags(self._m, C.byref(sc), C.byref(ce), C.byref(emin), C.byref(emax), _dp(ae)))
        return {"scalesf": bool(sc.value), "centersf": bool(ce.value), "emin": emin.value, "emax": emax.value,
                "atomenergies": ae}

    def symfunctions(self, z: int) -> np.ndarray:
        """sfLists(z): (nsf, 11) rows name, el1, el2, rcut, eta, lambda, zeta,
        Rs, sfmin, sfmax, sfmean in the reference's sorted order."""
        n = C.c_int()
        _check(lib().hdnnp_model_symfunctions(self._m, int(z), C.byref(n), None))
        out = np.zeros((n.value, 11))
        _check(lib().hdnnp_model_symfunctions(self._m, int(z), C.byref(n), _dp(out)))
        return out

    def network(self, z: int):
        """nnList(z): [(W (nout, nin), b (nout,), activation), ...]."""
        nl = C.c_int()
        _check(lib().hdnnp_model_network(self._m, int(z), C.byref(nl), None, None, None))
        dims = np.zeros(2 * nl.value, np.int32)
        acts = C.create_string_buffer(nl.value + 1)
        _check(lib().hdnnp_model_network(self._m, int(z), C.byref(nl), dims.ctypes.data_as(C.POINTER(C.c_int)),
                                         acts, None))
        total = sum(int(dims[2 * l]) * int(dims[2 * l + 1]) + int(dims[2 * l + 1]) for l in range(nl.value))
        vals = np.zeros(total)
        _check(lib().hdnnp_model_network(self._m, int(z), C.byref(nl), dims.ctypes.data_as(C.POINTER(C.c_int)),
                                         acts, _dp(vals)))
        out, o = [], 0
        for l in range(nl.value):
            nin, nout = int(dims[2 * l]), int(dims[2 * l + 1])
            W = vals[o:o + nin * nout].reshape(nin, nout).T.copy()  # Fortran (nout, nin) order
            o += nin * nout
            b = vals[o:o + nout].copy()
            o += nout
            out.append((W, b, acts.raw[l:l + 1].decode()))
        return out

    # ------------------------------------------------------------------ committee
    def committee_energy_and_forces(self, members: Sequence["Hdnnp"], ats: AtStruct, dEdLat: bool = False):
        """globalHdnnpEnergyAndForces (globalHdnnps.f90:31): members[0] must be
        this potential (it provides the symmetry functions).  Returns mean
        energy, mean forces (nat, 3), mean dE/dh (3, 3) or None, and the
        standard deviation of the member energies."""
        n = ats.nat
        E, sd = C.c_double(), C.c_double()
        F = np.zeros((n, 3))
        dl = np.zeros(9) if dEdLat else None
        arr = (C.c_void_p * len(members))(*[m._m for m in members])
        _check(lib().hdnnp_committee_energy_and_forces(
            self._c, arr, len(members), n, _ip(ats.el), _dp(ats.ats), 1 if ats.periodic else 0,
            _dp(_lat_flat(ats.lat)), C.byref(E), _dp(F), _dp(dl), C.byref(sd)))
        return E.value, F, (dl.reshape(3, 3, order="F") if dl is not None else None), sd.value

    def committee_eval_batch(self, members: Sequence["Hdnnp"], structs: Sequence[dict], dEdLat: bool = True):
        """Committee over a batch: dict of energy, forces, dEdLat, std."""
        off = np.zeros(len(structs) + 1, np.int64)
        off[1:] = np.cumsum([len(s["Z"]) for s in structs])
        Z = np.ascontiguousarray(np.concatenate([s["Z"] for s in structs]), dtype=np.int32)
        pos = np.ascontiguousarray(np.concatenate([s["pos"] for s in structs]), dtype=np.float64)
        lat = np.concatenate([_lat_flat(s["lat"]) for s in structs])
        per = np.array([0 if s["lat"] is None else 1 for s in structs], np.int32)
        ns = len(structs)
        out = {"energy": np.zeros(ns), "forces": np.zeros((int(off[-1]), 3)),
               "dEdLat": np.zeros(9 * ns) if dEdLat else None, "std": np.zeros(ns)}
        arr = (C.c_void_p * len(members))(*[m._m for m in members])
        _check(lib().hdnnp_committee_eval_batch(
            self._c, arr, len(members), ns, off.ctypes.data_as(C.POINTER(C.c_int64)), _ip(Z), _dp(pos), _ip(per),
            _dp(lat), _dp(out["energy"]), _dp(out["forces"]), _dp(out["dEdLat"]), _dp(out["std"])))
        return out

    def eval_batch_arrays(self, off, Z, pos, per, lat_flat, dEdLat=True, out=None):
        ns = len(off) - 1
        if out is None:
            out = {"energy": np.zeros(ns), "forces": np.zeros((int(off[-1]), 3)),
                   "dEdLat": np.zeros(9 * ns) if dEdLat else None}
        _check(lib().hdnnp_eval_batch(
            self._c, ns, off.ctypes.data_as(C.POINTER(C.c_int64)), _ip(Z), _dp(pos), _ip(per), _dp(lat_flat),
            _dp(out["energy"]), _dp(out["forces"]), _dp(out["dEdLat"])))
        return out

    STAGES = ("neighbour_count", "neighbour_fill", "element_groups", "sf_values", "mlp", "sf_gradients",
              "force_reduce")
    COUNTERS = ("evaluations", "atoms", "entries", "cand_pairs", "pairs", "g4_terms", "g2_terms")

    def set_profiling(self, on: bool = True):
        _check(lib().hdnnp_ctx_set_profiling(self._c, 1 if on else 0))

    def profile(self, reset: bool = False):
        ms = np.zeros(8)
        cnt = np.zeros(8, np.int64)
        _check(lib().hdnnp_profile_read(self._c, _dp(ms), cnt.ctypes.data_as(C.POINTER(C.c_int64)), 1 if reset else 0))
        return dict(zip(self.STAGES, ms[:7].tolist())), dict(zip(self.COUNTERS, cnt[:7].tolist()))

    def launches(self) -> int:
        n = C.c_int()
        _check(lib().hdnnp_last_launch_count(self._c, C.byref(n)))
        return n.value

    def fetch(self, what: str, count: int, dtype=np.float64):
        a = np.zeros(count, dtype=dtype)
        _check(lib().hdnnp_debug_fetch(self._c, what.encode(), a.ctypes.data_as(C.c_void_p), a.nbytes))
        return a


def dEdLat_to_stress(lat, dEdLat):
    """dEdLat2Stress (atomicStructure.f90:679): stress = -1/det(h) dEdLat h^T."""
    out = np.zeros(9)
    L = np.asarray(lat, dtype=np.float64).ravel(order="F").copy()
    dl = np.asarray(dEdLat, dtype=np.float64).ravel(order="F").copy()
    _check(lib().hdnnp_dEdLat_to_stress(_dp(L), _dp(dl), _dp(out)))
    return out.reshape(3, 3, order="F")


def debug_math(which: int, x) -> np.ndarray:
    """The branch-free FP64 exp (0), tanh on [0, 1] (1), sqrt (2) and 1/sqrt
    (3) of the symmetry-function kernels, evaluated on the current device."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    _check(lib().hdnnp_debug_math(which, x.size, _dp(x), _dp(y)))
    return y


def exported_symbols(header: str):
    """Function names declared in a C header (for the load test)."""
    import re

    txt = open(header).read()
    return sorted(set(re.findall(r"\b(hdnnp_[a-z0-9_]+)\s*\(", txt)))
