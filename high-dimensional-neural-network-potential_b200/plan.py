"""Resident plans over the C ABI (``hdnnp_plan_*`` in include/hdnnp_gpu.h).

A plan fixes a batch of structures and captures one evaluation -- or a
number of velocity-Verlet MD steps (src/potentials/hdnnpExample.f90:61-64) --
into a CUDA graph that ``launch()`` replays without host work.  Inputs and
results live in device memory (torch tensors are used only as the
allocator):

    p = Plan(pot, structs, precision=HDNNP_PREC_MIXED, skin=1.0,
             masses=m, momenta=p0, dt=20.0, steps_per_launch=10)
    p.launch(); builds = p.sync()
    E, F, dEdLat = p.results()

``structs`` is a list of dicts with ``Z``, ``pos`` (nat, 3) and ``lat``
(3, 3, columns = lattice vectors) or None for a molecule.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .engine import HDNNP_PREC_FP64, _check, lib


class _Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("margin", C.c_double), ("skin", C.c_double), ("momenta_dev", C.c_void_p),
                ("masses_dev", C.c_void_p), ("dt", C.c_double), ("steps_per_launch", C.c_int),
                ("energy_hist_dev", C.c_void_p), ("profile", C.c_int), ("autotune", C.c_int),
                ("single_block", C.c_int)]


def _register():
    L = lib()
    if getattr(L, "_plan_registered", False):
        return L
    P = C.c_void_p
    L.hdnnp_plan_create.argtypes = [P, P, C.c_int, P, P, P, P, P, P, P, P, C.POINTER(C.c_void_p)]
    L.hdnnp_plan_launch.argtypes = [P, P]
    L.hdnnp_plan_sync.argtypes = [P, P, C.POINTER(C.c_int64)]
    L.hdnnp_plan_info.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    L.hdnnp_plan_profile.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]
    L.hdnnp_plan_tuning.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.hdnnp_plan_free.argtypes = [P]
    L.hdnnp_plan_free.restype = None
    L._plan_registered = True
    return L


class Plan:
    def __init__(self, pot, structs, precision: int = HDNNP_PREC_FP64, margin: float = 0.25, skin: float = 0.0,
                 masses=None, momenta=None, dt: float = 0.0, steps_per_launch: int = 1, want_dEdLat: bool = True,
                 profile: bool = False, autotune: bool = False, single_block: bool = True):
        import torch

        L = _register()
        self._pot = pot  # the model must outlive the plan
        dev = torch.device("cuda", pot.device)
        self.nstruct = len(structs)
        off = np.zeros(self.nstruct + 1, np.int64)
        off[1:] = np.cumsum([len(s["Z"]) for s in structs])
        self.off = off
        self.natoms = int(off[-1])
        per = np.array([0 if s["lat"] is None else 1 for s in structs], np.int32)
        lat = np.concatenate([(np.eye(3) if s["lat"] is None else np.asarray(s["lat"], float)).ravel(order="F")
                              for s in structs])
        self.Z = torch.from_numpy(np.concatenate([np.asarray(s["Z"], np.int32) for s in structs])).to(dev)
        self.pos = torch.from_numpy(np.concatenate([np.asarray(s["pos"], float).reshape(-1, 3) for s in structs])).to(dev)
        self.E = torch.zeros(self.nstruct, dtype=torch.float64, device=dev)
        self.F = torch.zeros(self.natoms, 3, dtype=torch.float64, device=dev)
        self.L = torch.zeros(self.nstruct, 9, dtype=torch.float64, device=dev) if want_dEdLat else None
        self.mom = self.mass = self.hist = None
        if momenta is not None:
            self.mom = torch.from_numpy(np.asarray(momenta, float).reshape(-1, 3).copy()).to(dev)
            self.mass = torch.from_numpy(np.asarray(masses, float).copy()).to(dev)
            self.hist = torch.zeros(steps_per_launch, self.nstruct, dtype=torch.float64, device=dev)
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        self._opts = _Opts(int(precision), float(margin), float(skin), ptr(self.mom), ptr(self.mass), float(dt),
                           int(steps_per_launch), ptr(self.hist), 1 if profile else 0, 1 if autotune else 0,
                           0 if single_block else -1)
        self._per, self._lat = per, lat
        h = C.c_void_p()
        _check(L.hdnnp_plan_create(pot._m, C.byref(self._opts), self.nstruct, off.ctypes.data_as(C.c_void_p),
                                   per.ctypes.data_as(C.c_void_p), lat.ctypes.data_as(C.c_void_p), ptr(self.Z),
                                   ptr(self.pos), ptr(self.E), ptr(self.F), ptr(self.L), C.byref(h)))
        self._h = h

    def launch(self, stream=None):
        _check(lib().hdnnp_plan_launch(self._h, None if stream is None else C.c_void_p(stream)))

    def sync(self, stream=None) -> int:
        """Waits; raises HdnnpError on a device error; returns list builds."""
        n = C.c_int64()
        _check(lib().hdnnp_plan_sync(self._h, None if stream is None else C.c_void_p(stream), C.byref(n)))
        return n.value

    def info(self):
        e = C.c_int64()
        k = C.c_int()
        _check(lib().hdnnp_plan_info(self._h, C.byref(e), C.byref(k)))
        return {"entry_capacity": e.value, "kernels_per_launch": k.value}

    def tuning(self):
        """Launch shape chosen by the autotuner and its symmetry-function time."""
        a, b, t = C.c_int(), C.c_int(), C.c_double()
        _check(lib().hdnnp_plan_tuning(self._h, C.byref(a), C.byref(b), C.byref(t)))
        return {"sf_split": a.value, "sf_blocks_per_sm": b.value, "sf_ms": t.value}

    def profile(self, reset: bool = False):
        """(stage times in ms, work counters) as engine.Hdnnp.profile."""
        from .engine import Hdnnp

        ms = np.zeros(8)
        cnt = np.zeros(8, np.int64)
        _check(lib().hdnnp_plan_profile(self._h, ms.ctypes.data_as(C.POINTER(C.c_double)),
                                        cnt.ctypes.data_as(C.POINTER(C.c_int64)), 1 if reset else 0))
        return dict(zip(Hdnnp.STAGES, ms[:7].tolist())), dict(zip(Hdnnp.COUNTERS, cnt[:7].tolist()))

    def results(self):
        """(energies (nstruct,), forces (natoms, 3), dEdLat (nstruct, 3, 3) or None) as numpy."""
        E = self.E.cpu().numpy().copy()
        F = self.F.cpu().numpy().copy()
        D = None
        if self.L is not None:
            D = self.L.cpu().numpy().reshape(-1, 3, 3).transpose(0, 2, 1).copy()  # column-major rows
        return E, F, D

    def close(self):
        if getattr(self, "_h", None):
            lib().hdnnp_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
