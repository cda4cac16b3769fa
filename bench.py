#!/usr/bin/env python
"""Benchmark of the elastic contact solve on B200.

Workload (the single-solve non-periodic configuration): FreeFFTElasticHalfSpace
with a 1024 x 1024 topography, Hockney-padded to a 2048 x 2048 domain; seeded
self-affine Gaussian rough surface (Hurst 0.8, short-wavelength cutoff 4 px,
rolloff below 2 pi / (L/8), rms slope 0.1, L = 1, E* = 1); load sweep of 10
mean pressures log-spaced 1e-4 .. 1e-2 E*, each solve warm-started from the
previous displacement.  One step = one full sweep (10 solves).  Tolerances:
pentol = 1e-9 (max h - min h), forcetol = 1e-12 F, thermotol 1e-6.

Reported: solves/s of the mixed-precision path (FP32 bulk, FP64 reductions,
FP64 refinement) with inputs resident on the device (`value`); the plain FP64
path on the same sweep (`fp64_value`); the relative displacement error of the
mixed result against the FP64 result; p50 / p99 per-solve latency; `e2e`
through the public API with host (numpy) arrays; a roofline of the dominant
kernel from live CUDA-event timing; the CPU oracle on a bounded sample.
Further entries: `batched` (512 uneven periodic solves in one lockstep
batch), `serving` (the serving request mix -- sides 64..4096, 30 % free,
20 % plastic -- through ContactServer: closed-loop capacity, then an
open-loop Poisson stream at 80 % of it),
`plastic` (periodic 2048^2 with hardness, mixed vs FP64) and `operator` (the
standalone evaluate_disp against the HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CCG solves/s + p99 latency at 1e-6 rel err, mixed vs plain FP64, one B200"
N_TOPO = 1024
PRESSURES = np.logspace(-4, -2, 10)
SEED = 2026
WORKLOAD = ("free 1024x1024 topography (Hockney 2048x2048 domain), self-affine H=0.8 "
            "slope 0.1 cutoff 4px rolloff L/8, seed 2026; sweep of 10 mean pressures "
            "logspace(-4,-2) E*, warm-started; pentol 1e-9*(max h-min h), forcetol 1e-12*F")
CPU_BUDGET_S = 20.0
# Iterations of the FP64 solves of the sweep, load by load (the FP64 device
# path replays the reference's iteration sequence; the GPU arm re-measures
# them and reports both).  The CPU arms time a bounded sample of iterations
# and extrapolate to this count.
SWEEP_FP64_ITERS = (55, 61, 63, 73, 83, 89, 132, 197, 317, 431)
CONFIG = {"workload": WORKLOAD, "solves_per_step": 10,
          "l2": "256 MB buffer written between steps (> 126 MB L2)",
          "parallelism": "replicas"}


def surface():
    from contactmechanics_b200.Generation import self_affine
    return self_affine((N_TOPO, N_TOPO), (1.0, 1.0), 0.8, 0.1, seed=SEED,
                       rolloff_wavelength=1.0 / 8)


_SPANS = {}


def tolerances(h, F):
    """Solver tolerances of the sweep; the heights' span is computed once per array."""
    key = id(h)
    if key not in _SPANS:
        _SPANS[key] = (h, float(np.max(h) - np.min(h)))
    return dict(pentol=1e-9 * _SPANS[key][1], forcetol=1e-12 * F)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (numpy / scipy.fft with all host threads)
# ---------------------------------------------------------------------------
def cpu_sample(h, iters_per_load=6, substrate=None):
    """The oracle (numpy, scipy.fft on every host thread) on a bounded sample
    of the sweep: `iters_per_load` CCG iterations at the first and at the last
    load of the sweep (cold starts, so the second sample has the large
    contact area of the late loads), averaged into a cost per iteration and
    extrapolated to the sweep's full FP64 iteration count.  Returns solves/s
    of whole sweeps."""
    from oracle import contact_oracle as oc
    cores = os.cpu_count() or 1
    sub = substrate or oc.FreeSubstrate((N_TOPO, N_TOPO), 1.0, (1.0, 1.0), workers=cores)
    t0 = time.perf_counter()
    iters = 0
    for p in (PRESSURES[0], PRESSURES[-1]):
        r = oc.constrained_conjugate_gradients(sub, h, external_force=float(p),
                                               maxiter=iters_per_load, **tolerances(h, p))
        iters += r["nit"]
    el = time.perf_counter() - t0
    per_iter = el / iters
    sweep_s = per_iter * sum(SWEEP_FP64_ITERS)
    return dict(value=len(PRESSURES) / sweep_s, unit="solves/s", cores=cores, kind="port",
                sample=f"oracle (numpy, scipy.fft workers={cores}): {iters} CCG iterations "
                       f"({iters_per_load} at the first and at the last load, cold start) in "
                       f"{el:.1f} s = {per_iter * 1e3:.0f} ms/iteration, extrapolated to the "
                       f"sweep's {sum(SWEEP_FP64_ITERS)} FP64 iterations ({sweep_s:.0f} s per "
                       f"sweep of {len(PRESSURES)} solves)",
                seconds=el, iterations=iters, ms_per_iteration=per_iter * 1e3,
                sweep_seconds=sweep_s)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
def gpu_uuid(device_index):
    """nvidia-smi identifier (GPU-<uuid>) of CUDA device `device_index`."""
    import torch
    u = str(torch.cuda.get_device_properties(device_index).uuid)
    return u if u.startswith("GPU-") else "GPU-" + u


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        # nvidia-smi numbers GPUs in PCI order and ignores CUDA_VISIBLE_DEVICES,
        # so the timed GPU is selected by its UUID, not by the CUDA ordinal
        self.dev = gpu_uuid(device_index)
        self.samples = []
        self._p = None
        self._t = None
        self._first = threading.Event()

    def _read(self):
        for line in self._p.stdout:
            line = line.strip()
            if line:
                self.samples.append([x.strip() for x in line.split(",")])
                self._first.set()

    def __enter__(self):
        # one nvidia-smi process sampling every 200 ms, started before the
        # timed region (its start-up stays outside) and stopped after it
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._p = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        self._first.wait(5.0)
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            self._p.wait(timeout=5)
        except Exception:
            self._p.kill()
        self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "gpu": self.dev}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples), "gpu": self.dev}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def kernel_bytes(nx, ny, tx, ty, prec_bytes=4):
    """Compulsory bytes of each pass of the FP32 iteration: the solver fields
    (heights h, forces f, search direction t on the N topography points, the
    displacement u on the N_d domain points) and Green's tables each pass
    reads or writes, in the notation of the iteration's compulsory-byte model
    p (5 N + 2 N_d) + 2 p_t N_h.  The intermediate spectrum that passes hand
    to each other is not algorithmic traffic; it shows up in the measured
    DRAM traffic instead."""
    p = pt = prec_bytes
    N, Nd = tx * ty, nx * ny
    nh = nx * (ny // 2 + 1)
    return {
        "k_ccg_begin": 3 * p * N,          # f, u, h
        "k_ccg_gsum": 3 * p * N,           # f, u, h
        "k_row_fwd<T>": 5 * p * N,         # f, u, h, t in; t out
        "k_col<T>": pt * nh,               # Green's table
        "k_row_inv<T>": p * N,             # t
        "k_ccg_update": 5 * p * N,         # f, t, u, h in; f out
        "k_row_fwd<F>": 2 * p * N,         # f in and out
        "k_col<F>": pt * nh,               # Green's table
        # u in and out on the domain; h and both forces for the next
        # iteration's start statistics
        "k_row_inv<F>": 2 * p * Nd + 3 * p * N,
    }


def iteration_bytes(nx, ny, tx, ty, p=4, pt=4):
    """Compulsory bytes of one CCG iteration with state resident:
    p (5N + 2N_d) + 2 p_t N_h."""
    return p * (5 * tx * ty + 2 * nx * ny) + 2 * pt * nx * (ny // 2 + 1)


def load_traffic():
    path = os.path.join(ROOT, "profiles", "traffic_free1024.json")
    try:
        with open(path) as fh:
            return json.load(fh)
    except Exception:
        return {}


def run_gpu(args, rank, world, local_rank):
    import torch
    import contactmechanics_b200 as cm
    from contactmechanics_b200 import _lib
    from contactmechanics_b200.replicas import max_over_ranks
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    h = surface()
    hd = torch.from_numpy(h).cuda()
    sub = cm.FreeFFTElasticHalfSpace((N_TOPO, N_TOPO), 1.0, (1.0, 1.0))
    L = _lib.load_library()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def sweep(precision, host=False, lat=None):
        u0 = None
        out = []
        for p in PRESSURES:
            F = float(p)
            if lat is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
            r = cm.constrained_conjugate_gradients(
                sub, h if host else hd, external_force=F, precision=precision,
                initial_displacements=u0, **tolerances(h, F))
            if lat is not None:
                e1.record()
                e1.synchronize()
                lat.append(e0.elapsed_time(e1))
            if not r.success:
                raise RuntimeError(f"solve at p={F} did not converge: {r.message}")
            u0 = r.x
            out.append(r)
        return out

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(precision, steps, host=False, lat=None):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        res = None
        for _ in range(steps):
            flush.fill_(1.0)
            # the previous step's results go back to the allocator's cache
            # before this step allocates its own (else every other step pays
            # for fresh device allocations)
            res = None
            res = sweep(precision, host=host, lat=lat)
        e1.record()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist=dist, device="cuda")
        return ms, res

    for _ in range(args.warmup):
        sweep("mixed")
        sweep("fp64")
    # headline: mixed precision, device-resident inputs
    lat = []
    n0 = L.cm_launch_count()
    with ClockSampler(local_rank) as clocks:
        ms_mixed, res_mixed = timed("mixed", args.steps, lat=lat)
    launches = int(L.cm_launch_count() - n0)
    ms_fp64, res_fp64 = timed("fp64", args.steps)
    # end to end through the public API with host arrays
    sweep("mixed", host=True)
    ms_e2e, _ = timed("mixed", args.steps, host=True)

    solves = len(PRESSURES) * args.steps
    value = solves * world / (ms_mixed / 1e3)
    fp64_value = solves * world / (ms_fp64 / 1e3)
    e2e_value = solves * world / (ms_e2e / 1e3)
    n = N_TOPO
    errs, area_errs = [], []
    for a, b in zip(res_mixed, res_fp64):
        ua, ub = a.x[:n, :n], b.x[:n, :n]
        errs.append(float(torch.linalg.norm(ua - ub) / torch.linalg.norm(ub)))
        aa, ab = int((a.jac > 0).sum()), int((b.jac > 0).sum())
        area_errs.append(abs(aa - ab) / max(ab, 1))
    timing = {"mixed": [r.timing for r in res_mixed], "fp64": [r.timing for r in res_fp64]}
    iters = [r.nit for r in res_mixed]
    iters32 = [r.nit_fp32 for r in res_mixed]
    iters64 = [r.nit for r in res_fp64]

    # live per-kernel timing of the FP32 iteration (first load, cold start)
    P = _lib.CcgParams()
    P.precision = _lib.CM_FP32
    P.load_control = 1
    P.external_force = float(PRESSURES[0])
    tol = tolerances(h, float(PRESSURES[0]))
    P.pentol, P.forcetol, P.thermotol = tol["pentol"], tol["forcetol"], 1e-6
    P.mixfac, P.mixdecfac, P.minmixsteps, P.maxiter = 0.1, 0.95, 10, 100000
    ms_k = (ctypes.c_float * 16)()
    nk = ctypes.c_int()
    names = (ctypes.c_char_p * 16)()
    torch.cuda.synchronize()
    _lib.check(L.cm_ccg_profile(sub._plan.ptr, ctypes.byref(P), ctypes.c_void_p(hd.data_ptr()),
                                20, ms_k, ctypes.byref(nk), names))
    nxd, nyd = sub.nb_domain_grid_pts
    kb = kernel_bytes(nxd, nyd, n, n)
    per_kernel = {}
    for i in range(nk.value):
        name = names[i].decode()
        per_kernel[name] = {"ms": float(ms_k[i]), "bytes": kb.get(name)}
    dom = max(per_kernel, key=lambda k: per_kernel[k]["ms"])
    peak, peak_kind = peaks()
    t_dom = per_kernel[dom]["ms"] / 1e3
    achieved = per_kernel[dom]["bytes"] / t_dom / 1e9
    traffic = load_traffic().get(dom)
    t_iter = sum(v["ms"] for v in per_kernel.values()) / 1e3
    b_iter = iteration_bytes(nxd, nyd, n, n)
    # the FP32 iterations of the timed sweep as the solver runs them (CUDA
    # graphs, dependent launches): phase wall time over its iterations
    ms32 = sum(t["ms_fp32"] for t in timing["mixed"])
    t_iter_graph = ms32 / max(1, sum(iters32)) / 1e3
    return dict(
        value=value, ms_mixed=ms_mixed, fp64_value=fp64_value, ms_fp64=ms_fp64,
        e2e_value=e2e_value, ms_e2e=ms_e2e, lat=lat, launches=launches,
        clocks=clocks.summary(), rel_err=max(errs), area_err=max(area_errs),
        iters=iters, iters32=iters32, iters64=iters64, timing=timing,
        roofline={"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                  "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                  "traffic": traffic, "bytes_per_launch": per_kernel[dom]["bytes"],
                  "ms_per_launch": per_kernel[dom]["ms"]},
        iteration_roofline={"bytes": b_iter, "us_graph": t_iter_graph * 1e6,
                            "achieved_graph": b_iter / t_iter_graph / 1e9,
                            "frac_graph": b_iter / t_iter_graph / 1e9 / peak,
                            "us_eager_sum": t_iter * 1e6,
                            "frac_eager_sum": b_iter / t_iter / 1e9 / peak},
        per_kernel=per_kernel,
        h2d=h.nbytes + nxd * nyd * 8, d2h=nxd * nyd * 8 + h.nbytes + nxd * nyd)


# ---------------------------------------------------------------------------
# batched configuration: 512 independent periodic solves of uneven sizes
# ---------------------------------------------------------------------------
C3_SIDES = (64, 96, 128, 192, 256, 384, 512)
C3_N = 512
C3_WORKLOAD = ("512 periodic solves, nx, ny drawn uniformly from {64,96,128,192,256,384,512}, "
               "self-affine H~U[0.3,0.9], rms slope~U[0.05,0.2], mean pressure log-uniform "
               "1e-4..1e-2 E*, seed = index; pentol 1e-9*(max h-min h), forcetol 1e-12*F")


def c3_problems(n=C3_N):
    from contactmechanics_b200.Generation import self_affine
    probs = []
    for i in range(n):
        rng = np.random.default_rng(i)
        nx, ny = int(rng.choice(C3_SIDES)), int(rng.choice(C3_SIDES))
        hurst = rng.uniform(0.3, 0.9)
        slope = rng.uniform(0.05, 0.2)
        p = 10 ** rng.uniform(-4, -2)
        h = self_affine((nx, ny), (1.0, 1.0), hurst, slope, seed=i)
        probs.append(((nx, ny), h, float(p)))
    return probs


def run_batched(fp64_subset=48):
    """Mixed-precision batched solves/s of the 512-solve configuration, under
    the library's default launch shapes and under the autotuner's table
    (Autotune: tile sizes per side, block threads), the plain FP64
    single-solve path on a subset of the same solves, and the largest
    relative displacement difference between the two on that subset."""
    import torch
    import contactmechanics_b200 as cm
    from contactmechanics_b200 import Autotune
    probs = c3_problems()
    hs = [torch.from_numpy(h).cuda() for _, h, _ in probs]
    F = [p for _, _, p in probs]
    PT = [1e-9 * float(h.max() - h.min()) for _, h, _ in probs]
    FT = [1e-12 * p for p in F]

    def make_subs():
        # plans are created under the tuning in force
        return [cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0)) for nb, _, _ in probs]

    def timed_batch(subs):
        def batch():
            return cm.constrained_conjugate_gradients_batch(subs, hs, external_force=F, pentol=PT,
                                                            forcetol=FT, precision="mixed")
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = batch()
        e1.record()
        e1.synchronize()
        assert all(r.success for r in res)
        return res, e0.elapsed_time(e1)

    Autotune.clear()
    subs_default = make_subs()
    tuned = Autotune.load() if os.path.exists(Autotune.DEFAULT_TABLE) else None
    if tuned is not None:
        Autotune.apply(tuned)
    subs = make_subs()
    # one warm-up (allocations, graphs) of each, then alternating timed
    # batches, best of two each
    timed_batch(subs_default)
    timed_batch(subs)
    # a batch's results are released before the next timed batch allocates
    # its own (else that batch pays for fresh device allocations)
    ms_default = min(timed_batch(subs_default)[1] for _ in range(2))
    ms_batch, res = float("inf"), None
    for _ in range(2):
        res = None
        res, ms = timed_batch(subs)
        ms_batch = min(ms_batch, ms)
    # the same batch in one launch of the persistent cluster kernel (opt-in)
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    try:
        _lib.check(L.cm_tuning_set_batch_persistent(1))
        timed_batch(subs)
        ms_persistent = min(timed_batch(subs)[1] for _ in range(2))
    finally:
        L.cm_tuning_set_batch_persistent(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    idx = list(range(0, C3_N, C3_N // fp64_subset))[:fp64_subset]
    for i in idx:  # warm-up of the single-solve path: every plan's graphs captured
        cm.constrained_conjugate_gradients(subs[i], hs[i], external_force=F[i], pentol=PT[i],
                                           forcetol=FT[i], precision="fp64")
    torch.cuda.synchronize()
    e0.record()
    single = [cm.constrained_conjugate_gradients(subs[i], hs[i], external_force=F[i], pentol=PT[i],
                                                 forcetol=FT[i], precision="fp64") for i in idx]
    e1.record()
    e1.synchronize()
    ms_single = e0.elapsed_time(e1)
    errs = []
    for i, r in zip(idx, single):
        nb = subs[i].nb_grid_pts
        a, b = res[i].x[:nb[0], :nb[1]], r.x[:nb[0], :nb[1]]
        errs.append(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)))
    batched = C3_N / (ms_batch / 1e3)
    single_rate = len(idx) / (ms_single / 1e3)
    return {"workload": C3_WORKLOAD, "solves": C3_N,
            "mixed_batched_solves_per_s": batched, "ms_batch": ms_batch,
            "default_shapes_solves_per_s": C3_N / (ms_default / 1e3),
            "persistent_kernel_solves_per_s": C3_N / (ms_persistent / 1e3),
            "tuned_shapes": {k: tuned[k] for k in ("tiles", "threads")} if tuned else None,
            "fp64_single_solve_solves_per_s": single_rate,
            "fp64_single_solve_sample": f"{len(idx)} of the 512 solves (every {C3_N // fp64_subset}th)",
            "speedup_vs_fp64_single": batched / single_rate, "rel_err_vs_fp64_max": max(errs),
            "iterations_mean": float(np.mean([r.nit for r in res]))}


# ---------------------------------------------------------------------------
# C4 plastic solve and the standalone operator
# ---------------------------------------------------------------------------
C4_WORKLOAD = ("periodic 2048x2048, self-affine H=0.7 slope 0.2 seed 4, hardness 0.05 E*, mean "
               "pressure 5e-3 E*; pentol 1e-9*(max h-min h), forcetol 1e-9*F")


def run_plastic(reps=2):
    """Plastic configuration (C4): mixed vs FP64 solve, best of `reps`."""
    import torch
    import contactmechanics_b200 as cm
    from contactmechanics_b200.Generation import self_affine
    n = 2048
    h = self_affine((n, n), (1.0, 1.0), 0.7, 0.2, seed=4)
    hd = torch.from_numpy(h).cuda()
    sub = cm.PeriodicFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
    F = 5e-3
    kw = dict(external_force=F, hardness=0.05 / (n * n), pentol=1e-9 * float(h.max() - h.min()),
              forcetol=1e-9 * F, maxiter=20000)
    out, res = {"workload": C4_WORKLOAD}, {}
    for prec in ("mixed", "fp64"):
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = cm.constrained_conjugate_gradients(sub, hd, precision=prec, **kw)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        res[prec] = r
        out[prec] = {"solves_per_s": 1.0 / best, "ms": best * 1e3, "nit": r.nit,
                     "converged": bool(r.success)}
    a, b = res["mixed"], res["fp64"]
    out["rel_err_vs_fp64"] = float(torch.linalg.norm(a.x - b.x) / torch.linalg.norm(b.x))
    pa, pb = int(a.plastic.sum()), int(b.plastic.sum())
    ca, cb = int((a.jac > 0).sum()), int((b.jac > 0).sum())
    out["plastic_area_rel_err"] = abs(pa - pb) / max(pb, 1)
    out["contact_area_rel_err"] = abs(ca - cb) / max(cb, 1)
    out["plastic_fraction"] = pb / (n * n)
    out["speedup_vs_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    return out


def run_operator(reps=50):
    """The standalone operator (evaluate_disp, device-resident fields) on the
    C4 grid, the free 1024^2 grid and a periodic 3072^2 grid (sides 3 * 2^m):
    microseconds per call from CUDA events around `reps` back-to-back calls,
    and the operator's algorithmic bytes p (N + N_d) + p_t N_h against the
    measured HBM peak."""
    import torch
    import contactmechanics_b200 as cm
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    peak, peak_kind = peaks()
    out = {"workload": "evaluate_disp on device-resident fields; periodic 2048^2, free "
                       "1024^2 (2048^2 domain) and periodic 3072^2; cufft_us: torch.fft.rfft2 "
                       "x table x irfft2 (cuFFT) on the same fields", "peak_gbs": peak,
           "peak_source": peak_kind}
    for kind, n in (("periodic", 2048), ("free", 1024), ("periodic", 3072)):
        cls = cm.FreeFFTElasticHalfSpace if kind == "free" else cm.PeriodicFFTElasticHalfSpace
        sub = cls((n, n), 1.0, (1.0, 1.0))
        nxd, nyd = sub.nb_domain_grid_pts
        for prec in ("fp32", "fp64"):
            dt = torch.float32 if prec == "fp32" else torch.float64
            x = torch.randn((nxd, nyd), dtype=dt, device="cuda")
            y = torch.empty_like(x)
            stream = torch.cuda.current_stream()

            def call():
                _lib.check(L.cm_apply(sub._plan.ptr, _lib.CM_OP_DISP, _lib.PRECISIONS[prec],
                                      ctypes.c_void_p(x.data_ptr()), n if kind == "free" else nxd,
                                      n if kind == "free" else nyd, nyd, ctypes.c_void_p(y.data_ptr()),
                                      nxd, nyd, nyd,
                                      ctypes.c_void_p(stream.cuda_stream or _lib.CUDA_STREAM_LEGACY)))
            for _ in range(5):
                call()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                call()
            e1.record()
            torch.cuda.synchronize()
            us = e0.elapsed_time(e1) * 1e3 / reps
            p = 4 if prec == "fp32" else 8
            N = n * n
            b = p * (N + nxd * nyd) + p * nxd * (nyd // 2 + 1)
            gbs = b / us / 1e3
            # library baseline on the same box: cuFFT through torch.fft (R2C,
            # a separate multiply by the real table, C2R; zero padding by s=)
            xin = x[:n, :n].contiguous() if kind == "free" else x
            tab = torch.rand((nxd, nyd // 2 + 1), dtype=dt, device="cuda")

            def cufft():
                return torch.fft.irfft2(torch.fft.rfft2(xin, s=(nxd, nyd)) * tab, s=(nxd, nyd))
            for _ in range(5):
                cufft()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                cufft()
            e1.record()
            torch.cuda.synchronize()
            us_cufft = e0.elapsed_time(e1) * 1e3 / reps
            out[f"{kind}{n}_{prec}"] = {"us": us, "algorithmic_bytes": b, "GBps": gbs,
                                        "frac": gbs / peak, "cufft_us": us_cufft,
                                        "speedup_vs_cufft": us_cufft / us}
    return out


# ---------------------------------------------------------------------------
# serving: the request mix of the serving workload through the continuous-
# batching loop
# ---------------------------------------------------------------------------
# sides log-uniform 64..4096 rounded to the nearest size of this set (sides
# 2^k and 3 * 2^m, which the register-resident passes serve; a free 3072 side
# has a 6144-point domain)
C5_SIDES = (64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096)
C5_FREE_SIDES = C5_SIDES
C5_WORKLOAD = ("requests with side log-uniform 64..4096 rounded to {64,96,128,192,256,384,512,768,"
               "1024,1536,2048,3072,4096}; 30% free (domain x2), 20% plastic "
               "with hardness U[0.02,0.1] E*; mean pressure log-uniform 1e-4..1e-2 E*; self-affine "
               "H 0.8 slope 0.1 surfaces (8 seeds per side up to 1024, 2 above); pentol "
               "1e-9*(max h-min h), forcetol 1e-12*F (1e-9*F plastic); mixed precision")


def c5_requests(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        v = rng.uniform(np.log(64), np.log(4096))
        kind = "free" if rng.random() < 0.3 else "periodic"
        sides = C5_FREE_SIDES if kind == "free" else C5_SIDES
        side = min(sides, key=lambda x: abs(np.log(x) - v))
        plastic = rng.random() < 0.2
        hard = rng.uniform(0.02, 0.1) if plastic else None
        p = 10 ** rng.uniform(-4, -2)
        k = int(rng.integers(8 if side <= 1024 else 2))
        out.append((kind, side, k, p, hard))
    return out


def run_serving(n_requests=200, seed=7, **server_kw):
    """Capacity of the serving loop on `n_requests` requests of the serving
    mix (a closed loop: every request submitted at once), then the same
    requests as an open-loop Poisson stream at 80 % of that capacity: p50 /
    p99 latency from arrival to result, solves/s, and the largest relative
    displacement error of served results against the FP64 single-solve path
    on a sample.  Both runs serve the same requests, so the offered load is
    80 % of what the loop sustained on exactly that mix (the sizes are heavy
    tailed: a capacity taken on another sample can overstate it)."""
    import torch
    import contactmechanics_b200 as cm
    from contactmechanics_b200.Generation import self_affine
    from contactmechanics_b200.Serving import ContactServer
    surfaces = {}

    def surface(side, k):
        if (side, k) not in surfaces:
            surfaces[(side, k)] = torch.from_numpy(
                self_affine((side, side), (1.0, 1.0), 0.8, 0.1, seed=1000 * side + k)).cuda()
        return surfaces[(side, k)]

    def kwargs(side, h, p, hard):
        span = float(h.max() - h.min())
        kw = dict(external_force=p, pentol=1e-9 * span, forcetol=1e-12 * p, maxiter=20000)
        if hard is not None:
            kw["hardness"] = hard / (side * side)
            kw["forcetol"] = 1e-9 * p
        return kw

    srv = ContactServer(iters_per_step=8, **server_kw)
    # warm-up: one request of every kind and side, so plans, tables and kernels exist
    warm = []
    for kind, sides in (("periodic", C5_SIDES), ("free", C5_FREE_SIDES)):
        for side in sides:
            h = surface(side, 0)
            warm.append(srv.submit(kind, (side, side), (1.0, 1.0), h, external_force=1e-3,
                                   pentol=1e-6 * float(h.max() - h.min()), forcetol=1e-9))
    srv.start()
    for w in warm:
        w.done_event.wait(600)
    srv.completed.clear()
    torch.cuda.synchronize()

    def submit_all(reqs, arrivals, t0):
        handles = []
        for (kind, side, k, p, hard), at in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if at > now:
                time.sleep(at - now)
            h = surface(side, k)
            handles.append(srv.submit(kind, (side, side), (1.0, 1.0), h, arrival=t0 + at,
                                      **kwargs(side, h, p, hard)))
        for hd in handles:
            hd.done_event.wait(1200)
        return handles

    # closed loop: capacity
    reqs = c5_requests(n_requests, seed)
    t0 = time.perf_counter()
    cap_handles = submit_all(reqs, [0.0] * len(reqs), t0)
    t_cap = time.perf_counter() - t0
    capacity = len(reqs) / t_cap
    # open loop: the same requests, Poisson arrivals at 80 % of capacity
    rate = 0.8 * capacity
    rng = np.random.default_rng(seed + 1)
    reqs_open = list(reqs)
    rng.shuffle(reqs_open)
    n_open = len(reqs_open)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_open))
    t0 = time.perf_counter()
    handles = submit_all(reqs_open, arrivals, t0)
    t1 = time.perf_counter()
    srv.close()
    ok = [hd for hd in handles if hd.error is None and hd.result_value is not None]
    lat = np.array([hd.latency_s for hd in ok]) * 1e3
    # accuracy of served results against the FP64 single-solve path
    sample = [hd for hd in cap_handles if hd.error is None][:6]
    errs = []
    for hd in sample:
        sub = (cm.FreeFFTElasticHalfSpace if hd.kind == "free" else cm.PeriodicFFTElasticHalfSpace)(
            hd.nb_grid_pts, 1.0, (1.0, 1.0))
        r = cm.constrained_conjugate_gradients(sub, hd.heights, precision="fp64", **hd.solver_kwargs)
        n0, n1 = hd.nb_grid_pts
        a = np.asarray(hd.result_value.x)[:n0, :n1]
        b = r.x[:n0, :n1].cpu().numpy() if hasattr(r.x, "cpu") else r.x[:n0, :n1]
        errs.append(float(np.linalg.norm(a - b) / np.linalg.norm(b)))
    kinds = [r[0] for r in reqs_open]
    return {"workload": C5_WORKLOAD, "precision": "mixed",
            "capacity_solves_per_s": capacity, "capacity_requests": len(reqs),
            "capacity_s": t_cap, "capacity_failed": sum(hd.error is not None for hd in cap_handles),
            "offered_req_per_s": rate, "requests": n_open, "completed": len(ok),
            "converged": int(sum(bool(hd.result_value.success) for hd in ok)),
            "solves_per_s": len(ok) / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "rel_err_vs_fp64_max": max(errs) if errs else None, "rel_err_sample": len(errs),
            "free_fraction": kinds.count("free") / len(kinds),
            "target_req_per_s": 2000.0, "gap_to_target": 2000.0 / capacity}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the 512-solve batched configuration")
    ap.add_argument("--no-serving", action="store_true", help="skip the request-stream run")
    ap.add_argument("--no-plastic", action="store_true", help="skip the plastic configuration")
    ap.add_argument("--no-operator", action="store_true", help="skip the standalone operator")
    ap.add_argument("--profile-solve", choices=["mixed", "fp64", "fp32"], default=None,
                    help="run the first solve of the sweep once and exit (for profilers)")
    ap.add_argument("--profile-periodic", type=int, default=0,
                    help="with --profile-solve: a periodic N x N solve of a surface of the "
                         "sweep's kind instead (e.g. 3072 for the 3 * 2^m passes)")
    args = ap.parse_args()
    if args.profile_solve:
        import torch
        import contactmechanics_b200 as cm
        if args.profile_periodic:
            from contactmechanics_b200.Generation import self_affine
            n = args.profile_periodic
            h = self_affine((n, n), (1.0, 1.0), 0.8, 0.1, seed=SEED, rolloff_wavelength=1.0 / 8)
            sub = cm.PeriodicFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
        else:
            h = surface()
            sub = cm.FreeFFTElasticHalfSpace((N_TOPO, N_TOPO), 1.0, (1.0, 1.0))
        F = float(PRESSURES[0])
        # FP32 solves stop after 400 iterations: they need not reach the
        # sweep's FP64 tolerance, and a profiler needs only a few
        extra = {"maxiter": 400} if args.profile_periodic or args.profile_solve == "fp32" else {}
        r = cm.constrained_conjugate_gradients(sub, torch.from_numpy(h).cuda(), external_force=F,
                                               precision=args.profile_solve, **tolerances(h, F),
                                               **extra)
        torch.cuda.synchronize()
        print(json.dumps({"profile_solve": args.profile_solve, "nit": r.nit, "success": bool(r.success)}))
        return 0
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank != 0:
            return 0
        from oracle import contact_oracle as oc
        h = surface()
        cores = os.cpu_count() or 1
        sub = oc.FreeSubstrate((N_TOPO, N_TOPO), 1.0, (1.0, 1.0), workers=cores)
        for _ in range(args.warmup):
            cpu_sample(h, iters_per_load=1, substrate=sub)
        samples = [cpu_sample(h, iters_per_load=4, substrate=sub) for _ in range(args.steps)]
        ms_iter = float(np.median([x["ms_per_iteration"] for x in samples]))
        sweep_s = ms_iter / 1e3 * sum(SWEEP_FP64_ITERS)
        value = len(PRESSURES) / sweep_s
        ms_step = float(np.mean([x["seconds"] for x in samples])) * 1e3
        sample = (f"oracle (numpy, scipy.fft workers={cores}), FP64: each step times 8 CCG "
                  f"iterations (4 at the first and 4 at the last load of the sweep, cold start); "
                  f"median {ms_iter:.0f} ms/iteration over {args.steps} steps, extrapolated to "
                  f"the sweep's {sum(SWEEP_FP64_ITERS)} FP64 iterations ({sweep_s:.0f} s per "
                  f"sweep of {len(PRESSURES)} solves); ms_per_step is the sample's time")
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference", "config": dict(CONFIG),
                "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores,
                                 "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    r = run_gpu(args, rank, world, local_rank)
    batched = serving = plastic = operator = None
    if world == 1 and not args.no_operator:
        operator = run_operator()
    if world == 1 and not args.no_plastic:
        plastic = run_plastic()
    if world == 1 and not args.no_batched:
        batched = run_batched()
    if world == 1 and not args.no_serving:
        serving = run_serving()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        s = cpu_sample(surface())
        cpu = {k: s[k] for k in ("value", "unit", "cores", "kind", "sample")}
    lat = np.array(r["lat"])
    solves_per_step = len(PRESSURES)
    line = {
        "metric": METRIC, "value": r["value"], "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_mixed"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic", "config": dict(CONFIG),
        # precision-matched denominator and latency first, so a truncated
        # tail of the line keeps them
        "fp64_value": r["fp64_value"], "speedup_vs_fp64": r["value"] / r["fp64_value"],
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "rel_err_vs_fp64": r["rel_err"], "area_rel_err_vs_fp64": r["area_err"],
        "precision": "mixed: FP32 fields and transforms, FP64 reductions and scalars, FP64 "
                     "refinement iterations",
        "e2e": {"value": r["e2e_value"], "unit": "solves/s",
                "h2d_bytes_per_step": r["h2d"] * solves_per_step,
                "d2h_bytes_per_step": r["d2h"] * solves_per_step},
        "gpu_launches": r["launches"],
        "roofline": r["roofline"],
        "iteration_roofline": r["iteration_roofline"],
        "clocks": r["clocks"],
        "cpu_baseline": cpu,
        "iterations": {"mixed": r["iters"], "mixed_fp32_part": r["iters32"], "fp64": r["iters64"],
                       "fp64_reference_count": list(SWEEP_FP64_ITERS)},
        "per_kernel_ms": {k: v["ms"] for k, v in r["per_kernel"].items()},
        "operator": operator,
        "plastic": plastic,
        "batched": batched,
        "serving": serving,
        "latencies_ms": [round(float(x), 2) for x in lat],
        "solve_timing_ms": r["timing"],
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
