"""Serving form over the C ABI: continuous batching of MD / Monte Carlo walkers.

The reference drives one structure per ``hdnnpEnergyAndForces`` call from a
user-written MD loop (src/potentials/hdnnpExample.f90:59-72).  ``Server``
keeps many such trajectories ("walkers") resident on the GPU and evaluates
their requests in shared batches (``hdnnp_server_*`` in include/hdnnp_gpu.h):

    srv = Server(pot, max_batch_atoms=65536, workers=2, precision=HDNNP_PREC_MIXED)
    w = srv.add_walker(Z, pos, lat, masses=m, momenta=p)
    t = srv.submit(w, REQ_EVAL)
    E, F, dEdLat, latency_ms = srv.wait(t)
    t = srv.submit(w, REQ_MD_STEP, dt=20.0)      # hdnnpExample.f90:61-64 on the device

``pot`` is an ``engine.Hdnnp``; the server shares its model (the potential
must outlive the server).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from .engine import HDNNP_PREC_FP64, HdnnpError, _check, _dp, _ip, lib

REQ_EVAL = 0
REQ_MC_TRIAL = 1
REQ_MC_REJECT = 2
REQ_MD_STEP = 3
E_TIMEOUT = 4


class _Opts(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_batch_atoms", C.c_int), ("workers", C.c_int),
                ("precision", C.c_int), ("skin", C.c_double)]


class Server:
    def __init__(self, pot, max_batch_atoms: int = 65536, workers: int = 2, precision: int = HDNNP_PREC_FP64,
                 hbm_budget: int = 0, skin: float = 0.0):
        """skin > 0 (Bohr): walkers keep their neighbour lists (cutoff rc + skin)
        and build them again only after an atom moved by more than skin/2."""
        self._pot = pot  # keeps the model alive
        o = _Opts(int(hbm_budget), int(max_batch_atoms), int(workers), int(precision), float(skin))
        h = C.c_void_p()
        _check(lib().hdnnp_server_create(pot._m, C.byref(o), C.byref(h)))
        self._s = h
        self._nat = {}
        self._tw = {}  # ticket -> walker

    def close(self):
        if getattr(self, "_s", None):
            lib().hdnnp_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_walker(self, Z, pos, lat=None, masses=None, momenta=None) -> int:
        """A walker with atoms Z (nat,), positions (nat, 3); lat (3, 3) with
        lat[:, c] = lattice vector c, or None for a molecule."""
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        lf = None if lat is None else np.asarray(lat, dtype=np.float64).ravel(order="F").copy()
        m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
        p = None if momenta is None else np.ascontiguousarray(momenta, dtype=np.float64).reshape(-1, 3)
        w = C.c_int()
        _check(lib().hdnnp_server_add_walker(self._s, len(Z), _ip(Z), _dp(pos), 0 if lat is None else 1, _dp(lf),
                                             _dp(m), _dp(p), C.byref(w)))
        self._nat[w.value] = len(Z)
        return w.value

    def remove_walker(self, w: int):
        _check(lib().hdnnp_server_remove_walker(self._s, int(w)))
        self._nat.pop(w, None)

    def submit(self, w: int, kind: int = REQ_EVAL, dt: float = 0.0, sigma: float = 0.0, seed: int = 0) -> int:
        t = C.c_uint64()
        _check(lib().hdnnp_server_submit(self._s, int(w), int(kind), float(dt), float(sigma),
                                         int(seed) & 0xFFFFFFFFFFFFFFFF, C.byref(t)))
        self._tw[t.value] = w
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 600000):
        """(energy, forces (nat, 3), dEdLat (3, 3), latency_ms) of a finished
        request; raises HdnnpError (code E_TIMEOUT) if it is still running."""
        E = C.c_double()
        F = np.zeros((self._nat.get(self._tw.get(ticket), 0), 3))
        dl = np.zeros(9)
        lat = C.c_double()
        code = lib().hdnnp_server_wait(self._s, ticket, int(timeout_ms), C.byref(E), _dp(F), _dp(dl), C.byref(lat))
        if code != E_TIMEOUT:
            self._tw.pop(ticket, None)
        _check(code)
        return E.value, F, dl.reshape(3, 3, order="F"), lat.value

    def poll(self, ticket: int) -> Optional[tuple]:
        try:
            return self.wait(ticket, 0)
        except HdnnpError as e:
            if e.code == E_TIMEOUT:
                return None
            raise

    def next_done(self, timeout_ms: int = 1000) -> Optional[int]:
        """Ticket of the next finished request (completion order), or None."""
        t = C.c_uint64()
        code = lib().hdnnp_server_next_done(self._s, int(timeout_ms), C.byref(t))
        if code == E_TIMEOUT:
            return None
        _check(code)
        return t.value

    def read_walker(self, w: int):
        n = self._nat[w]
        pos = np.zeros((n, 3))
        mom = np.zeros((n, 3))
        _check(lib().hdnnp_server_read_walker(self._s, int(w), _dp(pos), _dp(mom)))
        return pos, mom

    def stats(self, reset: bool = False) -> dict:
        v = [C.c_double() for _ in range(4)]
        hbm = C.c_size_t()
        _check(lib().hdnnp_server_stats(self._s, *[C.byref(x) for x in v], C.byref(hbm), 1 if reset else 0))
        return {"p50_ms": v[0].value, "p99_ms": v[1].value, "atom_steps_per_s": v[2].value,
                "mean_batch_requests": v[3].value, "hbm_charged": hbm.value}

    def list_stats(self) -> dict:
        """Walker neighbour lists built and kept so far (skin > 0)."""
        b, k = C.c_int64(), C.c_int64()
        _check(lib().hdnnp_server_list_stats(self._s, C.byref(b), C.byref(k)))
        return {"built": b.value, "kept": k.value}


def poisson_load(srv: Server, walkers, rate: Optional[float], duration: float, seed: int = 0, sigma: float = 0.05,
                 dt: float = 20.0, kT: float = 1e-3):
    """Drives a server with walker steps arriving by a Poisson process.

    walkers: list of (walker id, nat, md[, init]) -- md walkers take velocity-Verlet
    steps (REQ_MD_STEP, dt), the others Metropolis Monte Carlo steps: a trial
    move (REQ_MC_TRIAL, sigma) accepted with probability
    min(1, exp(-dE / kT)), else undone by REQ_MC_REJECT.  Every walker must
    have been evaluated once (REQ_EVAL) before.  Arrivals come at `rate` per
    second (None: closed loop, every idle walker steps at once) for
    `duration` seconds; each goes to a walker drawn uniformly among the idle
    ones (a walker has one step in flight at a time), or waits on the client
    until one is idle.  Returns throughput and latency percentiles: "server"
    latency is submit -> completion, "client" latency arrival -> completion
    (includes waiting for an idle walker).  A step that fails on its
    walker's own input (HdnnpError with code 1 or 3, e.g. positions that an
    unstable trajectory made non-finite) is listed in "failed_walkers"; the
    walker then restarts from `init` (keyword arguments of add_walker; its
    new id replaces the old one in `walkers`) or, without `init`, leaves the
    load.
    """
    import time

    rng = np.random.default_rng(seed)
    idle = list(range(len(walkers)))
    energy = {}
    backlog = []  # arrival times waiting for an idle walker
    inflight = {}  # ticket -> (walker index, arrival time, "step" | "reject" | "restart")
    lat_srv, lat_cli = [], []
    failed = []
    atoms = 0
    accepted = trials = 0
    t0 = time.perf_counter()
    t_end = t0 + duration
    next_arrival = t0 + (rng.exponential(1.0 / rate) if rate else 0.0)
    while True:
        now = time.perf_counter()
        if now < t_end:
            if rate:
                while next_arrival <= now:
                    backlog.append(next_arrival)
                    next_arrival += rng.exponential(1.0 / rate)
            else:
                backlog.extend([now] * max(0, len(idle) - len(backlog)))
        elif not inflight:
            break
        while backlog and idle and now < t_end:
            k = idle.pop(int(rng.integers(len(idle))))
            wid, nat, md = walkers[k][:3]
            if md:
                t = srv.submit(wid, REQ_MD_STEP, dt=dt)
            else:
                t = srv.submit(wid, REQ_MC_TRIAL, sigma=sigma, seed=int(rng.integers(1 << 62)))
            inflight[t] = (k, backlog.pop(0), "step")
        wait_ms = 50 if not rate or now >= t_end else max(0, min(50, int((next_arrival - now) * 1e3)))
        t = srv.next_done(wait_ms)
        if t is None or t not in inflight:
            continue
        k, t_arr, what = inflight.pop(t)
        wid, nat, md = walkers[k][:3]
        try:
            E, F, dl, ms = srv.wait(t, 0)
        except HdnnpError as e:
            if e.code not in (1, 3):  # only a walker's own input or size may fail it
                raise
            failed.append((wid, str(e)))
            init = walkers[k][3] if len(walkers[k]) > 3 else None
            if init is None:
                continue  # the walker leaves the load
            # restart the trajectory from its initial state
            srv.remove_walker(wid)
            wid = srv.add_walker(**init)
            walkers[k] = (wid, nat, md, init)
            energy.pop(k, None)
            inflight[srv.submit(wid, REQ_EVAL)] = (k, t_arr, "restart")
            continue
        done = time.perf_counter()
        if what != "step":
            idle.append(k)
            continue
        atoms += nat
        lat_srv.append(ms)
        lat_cli.append((done - t_arr) * 1e3)
        if not md:
            trials += 1
            e_old = energy.get(k)
            if e_old is None or E <= e_old or rng.random() < np.exp(-(E - e_old) / kT):
                energy[k] = E
                accepted += 1
                idle.append(k)
            else:
                inflight[srv.submit(wid, REQ_MC_REJECT)] = (k, t_arr, "reject")
        else:
            idle.append(k)
    wall = time.perf_counter() - t0
    pct = lambda v, q: float(np.percentile(v, q)) if v else None
    return {"offered_steps_per_s": rate, "duration_s": wall, "steps": len(lat_srv),
            "steps_per_s": len(lat_srv) / wall, "atom_steps_per_s": atoms / wall,
            "p50_ms": pct(lat_srv, 50), "p99_ms": pct(lat_srv, 99),
            "client_p50_ms": pct(lat_cli, 50), "client_p99_ms": pct(lat_cli, 99),
            "mc_acceptance": accepted / trials if trials else None, "failed_walkers": failed}
