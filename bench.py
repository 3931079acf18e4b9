"""Benchmark: atom-steps/s of energy + forces + stress on one or more B200s.

A step is one evaluation (E, F, dE/dh of every structure) of the batched
mixed-size workload: 4096 independent periodic ABX3 supercells with nx, ny, nz
uniform in {1..4} (12-768 atoms, ~759k atoms), per-structure strain up to 5 %
and N(0, 0.15 Bohr) jitter (seed 4 + rank), synthetic 5-element potential with
280 symmetry functions per element and 280-25-25-1 networks
(tests/golden/abx3).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
  python bench.py --impl reference ...   # the reference's algorithm on the host cores

value  = atoms x steps / device time of the K steps (max over ranks), inputs
         resident in HBM, the batch as a resident plan (hdnnp_plan_*: one
         CUDA-graph launch per step, autotuned symmetry-function launches),
         default precision "fp64" (FP64 throughout, the arithmetic of the
         reference), so that the ratio to the reference arm compares equal
         arithmetic.
e2e    = the same plan with pinned host buffers: H2D of Z/positions and D2H
         of energies/forces/dE/dh inside every step (wall clock, the stream
         synchronised each step); e2e.eager_one_call is the same through the
         one-call eager path (hdnnp_eval_batch, host set-up in every call).
error_vs_oracle: the largest errors of the timed plan's results against the
         FP64 oracle on a seeded sample of 64 of its structures (and the same
         for the mixed-precision plan in config.compare).
config.compare: the mixed-precision form as a plan (FP32 symmetry
         functions, tensor-core networks, FP64 wrap/energy/virial) with its
         error against the oracle and its roofline, the eager batched path,
         the plain FP64 form (hdnnp_energy_and_forces, one structure per call,
         the reference's API) on a sample of the structures, both north-star
         ratios, the served walkers (mixed), and the single-structure legs
         (methylammonium MD, 768-atom cell, 49,152-atom MD) with the CPU
         stand-in beside each.
cpu_baseline / --impl reference: the oracle source (the reference's loops,
         OpenMP over atoms) built g++ -O3 -march=native -fopenmp on the host
         that runs the bench, on all its cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__  # noqa: E402

POT_DIR = os.path.join(ROOT, "tests", "golden", "abx3")
EXAMPLE_DIR = os.path.join(ROOT, "tests", "golden", "example")
METRIC = "atom-steps/s (E+F+stress)"
# MD time step of the served walkers (a.u.).  The random-init potential is
# stiff: velocity Verlet at the example's 20 a.u. heats its trajectories until
# positions become non-finite within a few hundred steps; at 0.5 a.u. the total
# energy stays bounded over thousands of steps.
DT_SYNTH = 0.5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--structs", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=256, help="structures in the CPU baseline sample")
    ap.add_argument("--error-sample", type=int, default=64, help="structures checked against the oracle")
    ap.add_argument("--plain-sample", type=int, default=512, help="structures timed through the plain per-structure API")
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="seconds per load point of the serving leg (0: skip)")
    ap.add_argument("--md", type=int, default=1, help="1: run the device-resident MD legs")
    ap.add_argument("--only-leg", choices=["c1", "c2", "c3"], default=None,
                    help="run one single-structure leg alone (C1 example MD, C2 768-atom cell, C3 49,152-atom MD) "
                         "and print its JSON: for profiling")
    ap.add_argument("--lean", action="store_true",
                    help="device-resident steps only (no e2e, comparisons, peaks or CPU baseline): for profiler runs")
    return ap.parse_args()


def max_over_ranks(x, world, device):
    """The largest of the ranks' values of x: a job of replicas is as fast as
    its slowest rank.  With one rank, x itself."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(atoms_per_rank, world, steps, seconds):
    """Whole-job atom-steps/s of `world` replicas that each evaluate their own
    batch of `atoms_per_rank` atoms `steps` times in `seconds` (the slowest
    rank's time)."""
    return atoms_per_rank * world * steps / seconds


def workload(W, n, seed):
    structs = W.config_c4(n_struct=n, seed=seed)
    off, Z, pos, lat, per = W.concat(structs)
    latf = np.concatenate([l.ravel(order="F") for l in lat])
    return structs, off, Z, pos, per, latf


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML every 20 ms (reads only), or nvidia-smi every 200 ms where
    the NVML bindings are missing."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        # the CUDA device index names a physical GPU through CUDA_VISIBLE_DEVICES
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
        self.idx = int(vis[gpu_index]) if gpu_index < len(vis) and vis[gpu_index].strip().isdigit() else gpu_index
        self.samples = []  # (sm MHz, max sm MHz, set of reason names)
        self.source = None
        self._stop = threading.Event()
        self._th = None

    def _nvml_loop(self):
        import pynvml as N

        N.nvmlInit()
        try:
            h = N.nvmlDeviceGetHandleByIndex(self.idx)
            mx = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            bits = (N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                    N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap)
            self.source = "nvml, every 20 ms"
            while not self._stop.is_set():
                sm = float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((sm, mx, {n for n, b in zip(self.NAMES, bits) if r & b}))
                self._stop.wait(0.02)
        finally:
            N.nvmlShutdown()

    def _smi_loop(self):
        q = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        self.source = "nvidia-smi, every 200 ms"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if out.returncode == 0 and len(f) >= 6:
                    self.samples.append((float(f[0]), float(f[1]),
                                         {n for n, v in zip(self.NAMES, f[2:6]) if v == "Active"}))
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        def run():
            try:
                self._nvml_loop()
            except Exception:
                self._smi_loop()

        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()

    def stop(self):
        self._stop.set()
        if self._th:
            self._th.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [x[0] for x in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": sorted(set().union(*[x[2] for x in self.samples])), "samples": len(self.samples),
                "source": self.source}


def measured_peaks(torch):
    """FP64 and FP32 (no TF32) GEMM throughput of this GPU via cuBLAS (TFLOP/s):
    the measured CUDA-core denominators for the symmetry-function kernels
    (MEASURED_PEAKS.json holds only HBM and bf16 tensor peaks)."""
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    for name, dt, n in (("fp64", torch.float64, 8192), ("fp32", torch.float32, 8192)):
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out[name] = 2 * n ** 3 / best / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = prev
    torch.cuda.empty_cache()
    return out


# Floating-point operations per work unit EXECUTED by the lambda x zeta x eta
# symmetry-function kernels for the (2 lambda, zeta {1,2,4,16}, 2 eta) grid of
# this potential, counted from csrc/symfn_fast.cu (add/mul = 1, FMA = 2,
# sqrt/exp/tanh/div = 1).  Units come from the engine's counters.  The
# product-space kernels execute about 9x fewer operations than the
# reference's per-function loops; the roofline is therefore stated with the
# algorithmic count below and the executed count beside it.
FLOPS_EXECUTED = {
    "sf_values": {"entries": 30, "pairs": 88, "g2_terms": 6},
    "sf_gradients": {"entries": 57, "pairs": 263, "g2_terms": 13},
}

# Algorithmic operations per work unit of the reference's path (one value +
# gradient evaluation), derived from the operation counts of
# calcAllSymmetryFunctions (symmetryFunctions.f90:201-305) and the
# contraction of hdnnpCalcNNs (hdnnps.f90:515-553): 30 per neighbour entry,
# 20 per radial term, 90 per contributing angular pair (r_jk < rc), 100 per
# angular term; the networks 4 x (multiply-adds of 280-25-25-1) = 30,600 per
# atom.  Pairs with r_jk >= rc add exact zeros in the reference and are not
# counted.
FLOPS_ALGORITHMIC = {"entries": 30, "g2_terms": 20, "pairs": 90, "g4_terms": 100}
MLP_FLOPS_PER_ATOM = 4 * (280 * 25 + 25 * 25 + 25)

# Algorithmic HBM bytes of the neighbour-list stages: positions and Z read
# once (28 B per atom), each entry (4 B index + 4 B image code) written once
# and read once (16 B per entry).
LIST_BYTES = {"atoms": 28, "entries": 16}


# DRAM bytes (read + write) per atom of each symmetry-function stage, from one
# ncu capture of both launches of each kernel on the first 1024 structures of
# this workload (191,160 atoms), scaled by the atoms of a step: the traffic of
# these kernels is per atom (positions, neighbour entries, G / dE/dG rows,
# pair lists), so it grows in proportion.
TRAFFIC_PER_ATOM = {"mixed": {"sf_values": 706.5e6 / 191160, "sf_gradients": 842.5e6 / 191160},
                    "fp64": {"sf_values": 903.737e6 / 191160, "sf_gradients": 1171.905e6 / 191160}}


def kernel_flops(stage, counters, evals):
    per = FLOPS_EXECUTED[stage]
    return sum(per[k] * counters[k] for k in per) / max(evals, 1)


def roofline(stage_ms, counters, peaks, precision, hbm_gbs):
    """Roofline of the symmetry-function passes (the dominant pair of kernels,
    k_sfv_fast + k_sfg_fast: ~80 % of a step), by the algorithmic count per
    launch pair, with the executed count, the whole step and the list stages
    beside it."""
    evals = max(counters["evaluations"], 1)
    per_step = {k: v / evals for k, v in counters.items() if k != "evaluations"}
    ms = {k: v / evals for k, v in stage_ms.items()}
    peak_key = "fp64" if precision == "fp64" else "fp32"
    peak = peaks.get(peak_key)
    sf_ms = ms["sf_values"] + ms["sf_gradients"]
    if not sf_ms > 0:
        return {"bound": peak_key + "-alu", "kernel": "sf_values + sf_gradients", "achieved": None, "peak": peak,
                "unit": "TFLOP/s", "frac": None, "note": "no stage times recorded"}
    alg = sum(FLOPS_ALGORITHMIC[k] * per_step[k] for k in FLOPS_ALGORITHMIC)
    achieved = alg / (sf_ms / 1e3) / 1e12
    step_ms = sum(ms.values())
    step_alg = alg + MLP_FLOPS_PER_ATOM * per_step["atoms"]
    list_ms = ms["neighbour_count"] + ms["neighbour_fill"]
    list_bytes = sum(LIST_BYTES[k] * per_step[k] for k in LIST_BYTES)
    executed = {}
    for k in ("sf_values", "sf_gradients"):
        f = kernel_flops(k, counters, evals)
        a = f / (ms[k] / 1e3) / 1e12
        executed[k] = {"flops_per_launch": f, "ms_per_launch": ms[k], "achieved_tflops": a,
                       "frac": a / peak if peak else None}
    tr = TRAFFIC_PER_ATOM.get(precision)
    traffic = sum(tr[k] for k in tr) * per_step["atoms"] if tr else None
    return {"bound": peak_key + "-alu", "kernel": "sf_values + sf_gradients (k_sfv_fast, k_sfg_fast)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            "flops_per_launch": alg, "ms_per_launch": sf_ms,
            "flops_source": "algorithmic: 30 per entry + 20 per radial term + 90 per contributing angular pair + "
                            "100 per angular term, times this step's unit counters",
            "peak_source": f"measured in this run: cuBLAS {peak_key.upper()} GEMM (no TF32), best of 5 (of measured)",
            "traffic": traffic, "traffic_unit": "bytes per step, DRAM read + write",
            "traffic_source": "ncu capture of the same kernels on 1024 of the structures, scaled by atoms"
            if traffic else "not captured for this precision",
            "executed": executed,
            "step": {"flops": step_alg, "ms": step_ms, "achieved_tflops": step_alg / (step_ms / 1e3) / 1e12,
                     "frac": step_alg / (step_ms / 1e3) / 1e12 / peak if peak else None},
            "lists": {"bytes": list_bytes, "ms": list_ms, "achieved_gbs": list_bytes / (list_ms / 1e3) / 1e9,
                      "peak_gbs": hbm_gbs, "frac": list_bytes / (list_ms / 1e3) / 1e9 / hbm_gbs if hbm_gbs else None,
                      "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm_gbs else None},
            "stage_ms_per_step": ms, "units_per_step": per_step}


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0  # fallback figure of this GPU pool


def oracle_errors(plan, structs, n, seed=8):
    """Largest errors of a plan's results against the FP64 oracle (checker
    build) on a seeded sample of its structures."""
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    model = O.Model(POT_DIR)
    E, F, D = plan.results()
    idx = np.sort(np.random.default_rng(seed).choice(len(structs), min(n, len(structs)), replace=False))
    out = {"dE_per_atom": 0.0, "dE_rel": 0.0, "dF_max": 0.0, "d_dEdLat_per_atom": 0.0, "d_dEdLat_max": 0.0}
    for k in idx:
        s = structs[int(k)]
        ref = model.eval(s["Z"], s["pos"], s["lat"])
        na = len(s["Z"])
        a0, a1 = plan.off[k], plan.off[k + 1]
        dE = abs(E[k] - ref["energy"])
        out["dE_per_atom"] = max(out["dE_per_atom"], dE / na)
        out["dE_rel"] = max(out["dE_rel"], dE / abs(ref["energy"]))
        out["dF_max"] = max(out["dF_max"], float(np.abs(F[a0:a1] - ref["forces"]).max()))
        dl = float(np.abs(D[k] - ref["dEdLat"]).max())
        out["d_dEdLat_per_atom"] = max(out["d_dEdLat_per_atom"], dl / na)
        out["d_dEdLat_max"] = max(out["d_dEdLat_max"], dl)
    out["sample"] = f"{len(idx)} of the batch's structures (seed {seed}), FP64 oracle"
    out["units"] = "Ha (energy), Ha/Bohr (forces), Ha (dE/dh)"
    return out


def cpu_baseline(structs, sample, seed=0):
    """The oracle source (the C++ restatement of the reference, OpenMP over
    atoms) built -O3 -march=native -fopenmp for this host, on all host
    threads, on a seeded sample of the workload's structures."""
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    m = O.Model(POT_DIR, native=True)
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(structs), size=min(sample, len(structs)), replace=False)
    atoms = 0
    t0 = time.perf_counter()
    for k in idx:
        s = structs[int(k)]
        m.eval(s["Z"], s["pos"], s["lat"])
        atoms += len(s["Z"])
    dt = time.perf_counter() - t0
    return {"value": atoms / dt, "unit": "atom-steps/s", "cores": O.max_threads(), "kind": "port",
            "build": O.NATIVE_FLAGS,
            "sample": f"{len(idx)} of the workload's structures ({atoms} atoms), one E+F+stress evaluation each, "
                      f"{dt:.1f} s"}


def run_reference(args, rank, world):
    """--impl reference: the reference's algorithm on the host cores.  The
    Fortran reference cannot be built in this image (no Fortran compiler), so
    its C++ restatement (the oracle: same loops, OpenMP over atoms), built
    -O3 -march=native -fopenmp on this host, runs it."""
    if rank != 0:
        return
    W = __graft_entry__.load_package().workloads
    structs, off, *_ = workload(W, args.structs, 4)
    steps = []
    base = None
    for it in range(args.warmup + args.steps):
        b = cpu_baseline(structs, max(8, args.cpu_sample // 4), seed=it)
        if it >= args.warmup:
            steps.append(b["value"])
        base = b
    v = float(np.mean(steps))
    line = {"metric": METRIC, "value": v, "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "batched mixed sizes: 4096 periodic ABX3 supercells (12-768 atoms), seed 4",
                       "step": "E+F+stress of a seeded sample of the structures (atom-steps/s is size-free)"},
            "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": base["cores"], "kind": "port",
                             "build": base["build"], "sample": base["sample"]},
            "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_leg(pkg, engine, pot, prec, seconds):
    """Served walkers: 256 ABX3 supercell walkers of 96-3072 atoms (seed 5),
    half velocity-Verlet MD (300 K, dt DT_SYNTH = 0.5 a.u.), half Metropolis MC
    (N(0, 0.05 Bohr) trial moves), resident on the device in one server
    (3 workers, 131,072-atom batches, 32 GB HBM budget).  A closed-loop
    point (every idle walker steps at once) gives the saturated throughput;
    Poisson arrivals at 25/50/80 % of it give latency under load."""
    from hdnnp_b200 import server as S

    W = pkg.workloads
    walkers = W.config_c5()
    budget = 32 << 30
    srv = S.Server(pot, max_batch_atoms=131072, workers=3, precision=prec, hbm_budget=budget)
    info = []
    for k, s in enumerate(walkers):
        md = k % 2 == 0
        m, p = W.maxwell_boltzmann(s["Z"], 300.0, 1000 + k) if md else (None, None)
        init = dict(Z=s["Z"], pos=s["pos"], lat=s["lat"], masses=m, momenta=p)
        info.append((srv.add_walker(**init), len(s["Z"]), md, init))
    ts = [srv.submit(w[0], S.REQ_EVAL) for w in info]
    for t in ts:
        srv.wait(t)
    S.poisson_load(srv, info, None, min(1.0, seconds), seed=50, dt=DT_SYNTH)  # warm-up (workspaces grow)
    srv.stats(reset=True)

    def point(rate, seed):
        r = S.poisson_load(srv, info, rate, seconds, seed=seed, dt=DT_SYNTH)
        r["mean_batch_requests"] = srv.stats(reset=True)["mean_batch_requests"]
        f = r.pop("failed_walkers")
        r["restarts"] = len(f)  # trajectories restarted after their positions became non-finite
        return r

    sat = point(None, 51)
    sweep = [point(frac * sat["steps_per_s"], 52 + k) for k, frac in enumerate((0.25, 0.5, 0.8))]
    hbm = srv.stats()["hbm_charged"]
    srv.close()
    nat = [w[1] for w in info]
    return {"workload": f"{len(info)} walkers, {min(nat)}-{max(nat)} atoms ({sum(nat)} total), half MD half MC",
            "server": "3 workers, 131072-atom batches", "hbm_budget": budget, "hbm_charged": hbm,
            "saturation": sat, "poisson_sweep": sweep}


def md_legs(pkg, engine, PLm, pot, torch, which=("c1", "c2", "c3")):
    """The single-structure workloads, each with the CPU stand-in (the oracle
    on all host threads) timed beside it.

    methylammonium: the reference's example (8 atoms, non-periodic, example
      potential, FP64), velocity Verlet at dt = 20 a.u. from seeded 140 K
      momenta: 1000 steps as 10 launches of a 100-step CUDA graph; per-step
      latency.  Beside it the same MD through the plain per-call API (host
      integrator, hdnnp_energy_and_forces every step), as the reference runs it.
    cell_768: the 768-atom cell, one evaluation per call (FP64 and mixed) and
      as a resident plan.
    strained_49152: 16x16x16 supercell of the ABX3 cell with a 3 % random
      triclinic strain (seed 2), Maxwell-Boltzmann 300 K (seed 3), 200 steps
      as 10 launches of 20, 1 Bohr Verlet skin, mixed precision, dt DT_SYNTH;
      the CPU stand-in runs the 8x8x8 cut of the same cell.
    """
    W = pkg.workloads
    out = {}

    st = torch.cuda.Stream()  # events and graph launches on one real stream (not the NULL stream)

    def timed(plan, launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(launches):
            plan.launch(st.cuda_stream)
        e1.record(st)
        builds = plan.sync(st.cuda_stream)
        return e0.elapsed_time(e1) / 1e3, builds

    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    if "c1" in which:
        out.update(leg_c1(W, engine, PLm, timed))
    if "c2" in which:
        out.update(leg_c2(W, engine, PLm, pot, timed, O))
    if "c3" in which:
        out.update(leg_c3(W, engine, PLm, pot, timed, O))
    return out


def leg_c1(W, engine, PLm, timed):
    """C1: the reference's example molecule, MD on the device vs the plain API and the CPU oracle."""
    out = {}
    s, m, p0 = W.config_c1(EXAMPLE_DIR)
    pot1 = engine.Hdnnp.from_runner(EXAMPLE_DIR)
    pl = PLm.Plan(pot1, [s], masses=m, momenta=p0, dt=20.0, steps_per_launch=100, want_dEdLat=False)
    timed(pl, 1)  # warm-up
    sec, _ = timed(pl, 10)
    # the same MD as a CUDA graph of the separate kernels (the general path)
    pg = PLm.Plan(pot1, [s], masses=m, momenta=p0, dt=20.0, steps_per_launch=100, want_dEdLat=False,
                  single_block=False)
    timed(pg, 1)
    gsec, _ = timed(pg, 10)
    g_kernels = pg.info()["kernels_per_launch"] / 100
    pg.close()
    ats = engine.AtStruct(s["Z"], s["pos"])
    E, F, _ = pot1.energy_and_forces(ats)
    x, p = s["pos"].copy(), p0.copy()
    nh = 200
    t0 = time.perf_counter()
    for _ in range(nh):
        x = x + p / m[:, None] * 20.0 + 0.5 * F / m[:, None] * 400.0
        Fl = F
        E, F, _ = pot1.energy_and_forces(engine.AtStruct(s["Z"], x))
        p = p + 10.0 * (F + Fl)
    hsec = time.perf_counter() - t0
    # the plain call alone: through the Python wrapper, and straight through
    # the C ABI with preallocated host buffers (the reference's call shape)
    ncall = 2000
    t0 = time.perf_counter()
    for _ in range(ncall):
        pot1.energy_and_forces(ats)
    wsec = (time.perf_counter() - t0) / ncall
    L = engine.lib()
    Zc = np.ascontiguousarray(s["Z"], np.int32)
    Xc = np.ascontiguousarray(s["pos"], np.float64)
    Ec, Fc = C.c_double(), np.zeros((len(Zc), 3))
    args = (pot1._c, len(Zc), Zc.ctypes.data_as(C.POINTER(C.c_int)),
            Xc.ctypes.data_as(C.POINTER(C.c_double)), 0, None, C.byref(Ec),
            Fc.ctypes.data_as(C.POINTER(C.c_double)), None)
    for _ in range(100):
        L.hdnnp_energy_and_forces(*args)
    t0 = time.perf_counter()
    for _ in range(ncall):
        L.hdnnp_energy_and_forces(*args)
    asec = (time.perf_counter() - t0) / ncall
    # CPU stand-in: the oracle (all host threads) running the same MD loop
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    om = O.Model(EXAMPLE_DIR)
    x, p, F = s["pos"].copy(), p0.copy(), om.eval(s["Z"], s["pos"], None, stress=False)["forces"]
    t0 = time.perf_counter()
    for _ in range(1000):
        x = x + p / m[:, None] * 20.0 + 0.5 * F / m[:, None] * 400.0
        Fl = F
        F = om.eval(s["Z"], x, None, stress=False)["forces"]
        p = p + 10.0 * (F + Fl)
    csec = time.perf_counter() - t0
    out["methylammonium_md"] = {
        "workload": "reference example MD: 8 atoms, FP64, dt 20 a.u., 1000 steps (10 launches of 100; "
                    "one thread block runs all 100 steps of a launch)",
        "steps_per_s": 1000 / sec, "us_per_step": sec / 1000 * 1e6,
        "kernels_per_step": pl.info()["kernels_per_launch"] / 100,
        "graph_us_per_step": gsec / 1000 * 1e6, "graph_kernels_per_step": g_kernels,
        "plain_api_steps_per_s": nh / hsec, "plain_api_us_per_step": hsec / nh * 1e6,
        "plain_call_us": {"python_wrapper": wsec * 1e6, "c_abi": asec * 1e6,
                          "what": "one hdnnp_energy_and_forces on the 8-atom molecule, host arrays in and out, "
                                  "mean of 2000 back-to-back calls"},
        "cpu_oracle_steps_per_s": 1000 / csec, "cpu_cores": O.max_threads()}
    pl.close()
    pot1.close()
    return out


def leg_c2(W, engine, PLm, pot, timed, O):
    """C2: the 768-atom cell, one structure per call (FP64 and mixed) and as a plan (graph)."""
    out = {}
    s2 = W.config_c2()
    ats2 = engine.AtStruct(s2["Z"], s2["pos"], s2["lat"])
    c2 = {"workload": "768-atom ABX3 4x4x4 cell (seed 1), E+F+stress"}
    for name, prec in (("fp64", engine.HDNNP_PREC_FP64), ("mixed", engine.HDNNP_PREC_MIXED)):
        pot.set_precision(prec)
        pot.energy_and_forces(ats2, dEdLat=True)
        ts = []
        for _ in range(20):
            t0 = time.perf_counter()
            pot.energy_and_forces(ats2, dEdLat=True)
            ts.append(time.perf_counter() - t0)
        c2[f"plain_api_{name}_ms"] = float(np.median(ts) * 1e3)
        p2 = PLm.Plan(pot, [s2], precision=prec)
        timed(p2, 2)
        sec, _ = timed(p2, 20)
        c2[f"plan_{name}_ms"] = sec / 20 * 1e3
        p2.close()
    pot.set_precision(engine.HDNNP_PREC_FP64)
    om2 = O.Model(POT_DIR)
    om2.eval(s2["Z"], s2["pos"], s2["lat"])
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        om2.eval(s2["Z"], s2["pos"], s2["lat"])
        ts.append(time.perf_counter() - t0)
    c2["cpu_oracle_ms"] = float(np.median(ts) * 1e3)
    c2["atom_steps_per_s"] = {k[:-3]: 768 / (v / 1e3) for k, v in c2.items() if k.endswith("_ms")}
    out["cell_768"] = c2
    return out


def leg_c3(W, engine, PLm, pot, timed, O):
    """C3: the strained 49,152-atom cell, MD on the device with a 1 Bohr Verlet skin."""
    out = {}
    om2 = O.Model(POT_DIR)
    s3 = W.config_c3()
    m3, p3 = W.maxwell_boltzmann(s3["Z"], 300.0, 3)
    pl3 = PLm.Plan(pot, [s3], precision=engine.HDNNP_PREC_MIXED, skin=1.0, masses=m3, momenta=p3, dt=DT_SYNTH,
                   steps_per_launch=20, want_dEdLat=False)
    timed(pl3, 1)
    sec, builds = timed(pl3, 10)
    nat = len(s3["Z"])
    # CPU stand-in on the 8x8x8 cut of the same strained cell (per-atom rate)
    s3c = W.config_c3(n=8)
    om2.eval(s3c["Z"], s3c["pos"], s3c["lat"])
    t0 = time.perf_counter()
    for _ in range(2):
        om2.eval(s3c["Z"], s3c["pos"], s3c["lat"])
    c3sec = (time.perf_counter() - t0) / 2
    out["strained_49152_md"] = {
        "workload": f"{nat} atoms, 3% triclinic strain, 300 K, 200 MD steps (10 graph launches of 20), "
                    f"1 Bohr Verlet skin, mixed precision, dt {DT_SYNTH} a.u.",
        "atom_steps_per_s": nat * 200 / sec, "ms_per_step": sec / 200 * 1e3, "list_builds": builds,
        "cpu_oracle_atom_steps_per_s": len(s3c["Z"]) / c3sec,
        "cpu_sample": f"8x8x8 cut ({len(s3c['Z'])} atoms), E+F+stress, FP64"}
    pl3.close()
    pot.set_precision(engine.HDNNP_PREC_FP64)
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pkg = __graft_entry__.load_package()
    from hdnnp_b200 import engine

    W = pkg.workloads
    if args.only_leg:
        from hdnnp_b200 import plan as PLm

        pot = engine.Hdnnp.from_runner(POT_DIR, device=local)
        res = md_legs(pkg, engine, PLm, pot, torch, which=(args.only_leg,))
        if rank == 0:
            print(json.dumps({"leg": args.only_leg, **res}), flush=True)
        pot.close()
        return
    structs, off, Z, pos, per, latf = workload(W, args.structs, 4 + rank)
    natoms = int(off[-1])
    nstruct = len(structs)
    pot = engine.Hdnnp.from_runner(POT_DIR, device=local)
    prec = engine.HDNNP_PREC_MIXED if args.precision == "mixed" else engine.HDNNP_PREC_FP64
    pot.set_precision(prec)
    L = engine.lib()

    # device-resident inputs / outputs (torch only as the allocator)
    Zd = torch.from_numpy(Z).cuda()
    posd = torch.from_numpy(pos).cuda()
    Ed = torch.zeros(nstruct, dtype=torch.float64, device="cuda")
    Fd = torch.zeros(natoms, 3, dtype=torch.float64, device="cuda")
    Ld = torch.zeros(nstruct, 9, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()  # a real stream handle (the legacy default stream is NULL)

    def step_eager():
        # hdnnp_eval_batch_device: host set-up and one host read of the entry total per step
        engine._check(L.hdnnp_eval_batch_device(
            pot._c, nstruct, off.ctypes.data_as(C.POINTER(C.c_int64)), None, C.c_void_p(Zd.data_ptr()),
            C.c_void_p(posd.data_ptr()), per.ctypes.data_as(C.POINTER(C.c_int32)),
            latf.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(Ed.data_ptr()), C.c_void_p(Fd.data_ptr()),
            C.c_void_p(Ld.data_ptr()), C.c_void_p(stream.cuda_stream)))

    # the batch as a resident plan: one CUDA-graph launch per step, no host work
    from hdnnp_b200 import plan as PLm

    # autotuned launch shape of the symmetry-function kernels (before timing)
    bplan = PLm.Plan(pot, structs, precision=prec, margin=0.02, profile=True, autotune=True)

    def step_device():
        bplan.launch(stream.cuda_stream)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_device_steps(nsteps, fn=None, plan=None):
        times = []
        for _ in range(nsteps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            (fn or step_device)()
            e1.record(stream)
            times.append((e0, e1))
            if plan is not None:
                plan.sync(stream.cuda_stream)  # collects the stage events of this launch (outside e0..e1)
        return times

    # ---------------- value: inputs resident in HBM
    for _ in range(args.warmup):
        step_device()
    bplan.sync(stream.cuda_stream)
    bplan.profile(reset=True)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    torch.cuda.nvtx.range_push("bench_timed")  # profilers select the timed launches by this range
    times = timed_device_steps(args.steps, plan=bplan)
    torch.cuda.nvtx.range_pop()
    barrier()
    clk = clocks.stop()
    stage_ms, counters = bplan.profile(reset=True)
    dev_s = sum(a.elapsed_time(b) for a, b in times) / 1e3
    launches_per_step = bplan.info()["kernels_per_launch"]
    dev_s = max_over_ranks(dev_s, world, "cuda")
    value = weak_value(natoms, world, args.steps, dev_s)
    if args.lean:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "ms_per_step": dev_s / args.steps * 1e3,
                              "precision": args.precision, "stage_ms": stage_ms, "counters": counters,
                              "lean": True}), flush=True)
        bplan.close()
        pot.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # ---------------- e2e: pinned host buffers, copies inside every step.
    # Through the resident plan (hdnnp_plan_launch): each step copies the
    # batch's Z and positions in from pinned host memory, launches the graph
    # and copies energies, forces and dE/dh back, then waits for the stream.
    # The eager one-call path (hdnnp_eval_batch, host set-up and a host read
    # inside every call) is reported beside it as e2e_eager.
    Zh = torch.from_numpy(Z).pin_memory()
    posh = torch.from_numpy(pos).pin_memory()
    Eh = torch.zeros(nstruct, dtype=torch.float64).pin_memory()
    Fh = torch.zeros(natoms * 3, dtype=torch.float64).pin_memory()
    Lh = torch.zeros(nstruct * 9, dtype=torch.float64).pin_memory()
    dp = lambda x: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_double))

    def step_host():
        engine._check(L.hdnnp_eval_batch(
            pot._c, nstruct, off.ctypes.data_as(C.POINTER(C.c_int64)),
            C.cast(C.c_void_p(Zh.data_ptr()), C.POINTER(C.c_int32)), dp(posh),
            per.ctypes.data_as(C.POINTER(C.c_int32)), latf.ctypes.data_as(C.POINTER(C.c_double)),
            dp(Eh), dp(Fh), dp(Lh)))

    def step_host_plan():
        with torch.cuda.stream(stream):
            bplan.Z.copy_(Zh, non_blocking=True)
            bplan.pos.copy_(posh.view(bplan.pos.shape), non_blocking=True)
        bplan.launch(stream.cuda_stream)
        with torch.cuda.stream(stream):
            Eh.copy_(bplan.E, non_blocking=True)
            Fh.copy_(bplan.F.view(-1), non_blocking=True)
            Lh.copy_(bplan.L.view(-1), non_blocking=True)
        stream.synchronize()

    def wall(fn, n):
        barrier()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()  # returns after this step's D2H copies completed
        barrier()
        return max_over_ranks(time.perf_counter() - t0, world, "cuda")

    for _ in range(max(1, args.warmup // 2)):
        step_host_plan()
        step_host()
    e2e = weak_value(natoms, world, args.steps, wall(step_host_plan, args.steps))
    bplan.sync(stream.cuda_stream)  # device flags of the e2e steps (raises on an error)
    bplan.profile(reset=True)
    e2e_eager = weak_value(natoms, world, args.steps, wall(step_host, args.steps))
    h2d = Z.nbytes + pos.nbytes
    d2h = (Eh.numel() + Fh.numel() + Lh.numel()) * 8

    # ---------------- comparisons on the same workload (rank 0)
    compare = {}
    errors = {}
    peaks = measured_peaks(torch) if rank == 0 else {}
    hbm = hbm_peak()
    if rank == 0:
        errors[args.precision] = oracle_errors(bplan, structs, args.error_sample)
        nk = max(2, args.steps // 3)
        # the same precision without the graph (host set-up + one host read per step)
        step_eager()
        torch.cuda.synchronize()
        et = timed_device_steps(nk, fn=step_eager)
        torch.cuda.synchronize()
        compare["batched_eager_" + args.precision] = natoms * len(et) / (sum(a.elapsed_time(b) for a, b in et) / 1e3)
        # the other precision, as an autotuned plan, with its own roofline and error
        other = engine.HDNNP_PREC_FP64 if prec == engine.HDNNP_PREC_MIXED else engine.HDNNP_PREC_MIXED
        oname = "fp64" if other == engine.HDNNP_PREC_FP64 else "mixed"
        oplan = PLm.Plan(pot, structs, precision=other, margin=0.02, profile=True, autotune=True)
        for _ in range(args.warmup):
            oplan.launch(stream.cuda_stream)
        oplan.sync(stream.cuda_stream)
        oplan.profile(reset=True)
        ot = timed_device_steps(max(nk, args.steps // 2), fn=lambda: oplan.launch(stream.cuda_stream), plan=oplan)
        oplan.sync(stream.cuda_stream)
        osec = sum(a.elapsed_time(b) for a, b in ot) / 1e3
        ost, ocnt = oplan.profile(reset=True)
        compare["batched_" + oname] = natoms * len(ot) / osec
        compare["batched_" + oname + "_ms_per_step"] = osec / len(ot) * 1e3
        compare["batched_" + oname + "_roofline"] = roofline(ost, ocnt, peaks, oname, hbm)
        compare["batched_" + oname + "_autotuned"] = oplan.tuning()
        errors[oname] = oracle_errors(oplan, structs, args.error_sample)
        oplan.close()
        pot.set_precision(engine.HDNNP_PREC_FP64)
        rng = np.random.default_rng(7)
        idx = rng.choice(nstruct, size=min(args.plain_sample, nstruct), replace=False)
        sample = [engine.AtStruct(structs[int(k)]["Z"], structs[int(k)]["pos"], structs[int(k)]["lat"]) for k in idx]
        pot.energy_and_forces(sample[0], dEdLat=True)
        atoms = sum(a.nat for a in sample)
        t0 = time.perf_counter()
        for a in sample:
            pot.energy_and_forces(a, dEdLat=True)
        psec = time.perf_counter() - t0
        compare["plain_fp64_per_structure"] = atoms / psec
        compare["plain_sample"] = f"{len(sample)} structures ({atoms} atoms), hdnnp_energy_and_forces with host arrays"
        mixed_v = value if args.precision == "mixed" else compare["batched_mixed"]
        fp64_v = value if args.precision == "fp64" else compare["batched_fp64"]
        compare["speedup_ratios"] = {
            "target": "batched/served mixed >= 5x the plain FP64 GPU path on the same mixed-size workload",
            "mixed_over_plain_fp64_per_structure": mixed_v / compare["plain_fp64_per_structure"],
            "mixed_over_batched_fp64": mixed_v / fp64_v,
            "batched_fp64_over_plain_fp64_per_structure": fp64_v / compare["plain_fp64_per_structure"]}
        pot.set_precision(prec)
        if world == 1 and args.serve_seconds > 0:
            pot.set_precision(engine.HDNNP_PREC_MIXED)
            compare["served"] = serve_leg(pkg, engine, pot, engine.HDNNP_PREC_MIXED, args.serve_seconds)
            compare["served"]["precision"] = "mixed"
            compare["speedup_ratios"]["served_mixed_over_plain_fp64_per_structure"] = (
                compare["served"]["saturation"]["atom_steps_per_s"] / compare["plain_fp64_per_structure"])
            pot.set_precision(prec)
        if world == 1 and args.md:
            compare.update(md_legs(pkg, engine, PLm, pot, torch))

    # ---------------- roofline of the dominant kernels (the two SF passes)
    roof = roofline(stage_ms, counters, peaks, args.precision, hbm)

    if world > 1:
        dist.barrier()
    if rank == 0:
        cpu = cpu_baseline(structs, args.cpu_sample) if world == 1 else None
        line = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32 (f64 wrap/energy/virial)",
                "data": "synthetic (seeded ABX3 supercells, random-init 280-SF potential)",
                "config": {"workload": f"batched mixed sizes: {nstruct} periodic ABX3 supercells per GPU "
                                       f"(12-768 atoms, {natoms} atoms, seed 4+rank), E+F+stress",
                           "global_batch": natoms * world, "precision": args.precision,
                           "parallelism": f"replicas x{world} (independent structures per GPU)",
                           "autotuned": bplan.tuning(),
                           "l2": "256 MB buffer written between timed steps; working set (G alone "
                                 f"{natoms * 280 * (8 if args.precision == 'fp64' else 4) / 1e9:.1f}+ GB) "
                                 "is larger than L2",
                           "compare": compare},
                "error_vs_oracle": errors,
                "e2e": {"value": e2e, "unit": "atom-steps/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h),
                        "path": "resident plan: H2D of Z and positions, graph launch, D2H of E, F, dE/dh",
                        "eager_one_call": e2e_eager},
                "gpu_launches": launches_per_step * args.steps,
                "roofline": roof, "clocks": clk, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    bplan.close()
    pot.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
