"""Autotuner of the batched solver's launch shapes.

Batched solves (``constrained_conjugate_gradients_batch``) and the serving
loop run the per-pass kernels over a combined (solve, tile) work list; how
many transform elements a tile holds (per sequence length) and how many
threads a transform block has decide how well those launches fill the GPU.
``tune_batch`` measures them on the device: it solves one batch of seeded
rough periodic problems whose sides are drawn from the batched workload's
mix for a fixed number of iterations, and by coordinate descent keeps, for
every side (sequence length) in turn, the candidate tile size that makes
the whole batch fastest, then the block threads of the batched launches.
The choice is a JSON table (``save`` / ``load``);
``apply`` hands it to the library (``cm_tuning_*``), for plans created
afterwards.  The package ships the table measured on a B200
(``tuning/b200_batch.json``), which ``apply_default`` loads.
"""
import json
import os
import time

import numpy as np

from . import _lib

SIDES = (64, 96, 128, 192, 256, 384, 512)
TILE_CANDIDATES = {"fp32": (1024, 2048, 4096), "fp64": (512, 1024, 2048)}
THREAD_CANDIDATES = (128, 256, 512)
DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning",
                             "b200_batch.json")

_applied = False


def apply(table):
    """Install a tuning table {"tiles": {prec: {length: elems}}, "threads":
    {prec: threads}, "batch_persistent": bool} for plans created afterwards
    ("batch_persistent" selects the persistent cluster kernel for elastic
    batches instead of the lockstep graph)."""
    L = _lib.load_library()
    if "batch_persistent" in table:
        _lib.check(L.cm_tuning_set_batch_persistent(int(bool(table["batch_persistent"]))))
    for prec, tiles in table.get("tiles", {}).items():
        for length, elems in tiles.items():
            _lib.check(L.cm_tuning_set_tiles(_lib.PRECISIONS[prec], int(length), int(elems)))
    for prec, threads in table.get("threads", {}).items():
        _lib.check(L.cm_tuning_set_batch_threads(_lib.PRECISIONS[prec], int(threads)))


def clear(lengths=SIDES):
    """Back to the library's defaults."""
    L = _lib.load_library()
    _lib.check(L.cm_tuning_set_batch_persistent(0))
    for prec in ("fp32", "fp64"):
        for n in lengths:
            _lib.check(L.cm_tuning_set_tiles(_lib.PRECISIONS[prec], int(n), 0))
        _lib.check(L.cm_tuning_set_batch_threads(_lib.PRECISIONS[prec], 256))


def load(path=DEFAULT_TABLE):
    with open(path) as fh:
        return json.load(fh)


def save(table, path):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)


def apply_default():
    """Install the shipped table once (no-op when it is absent)."""
    global _applied
    if _applied:
        return
    _applied = True
    if os.path.exists(DEFAULT_TABLE):
        apply(load(DEFAULT_TABLE))


def _mix(sides, n, seed):
    """n problem shapes (nx, ny) with sides drawn uniformly from `sides`."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice(sides)), int(rng.choice(sides))) for _ in range(n)]


def _batch_seconds(shapes, precision, iters, seed, reps=3):
    """Seconds per iteration of a batch of seeded periodic solves of the given
    shapes stopped at `iters` iterations (plans created under the tuning in
    force)."""
    import torch
    from .FFTElasticHalfSpace import PeriodicFFTElasticHalfSpace
    from .Generation import self_affine
    from .Optimization import constrained_conjugate_gradients_batch
    subs, hs, F, PT = [], [], [], []
    for i, nb in enumerate(shapes):
        h = self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=seed + i)
        subs.append(PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0)))
        hs.append(torch.from_numpy(h).cuda())
        F.append(3e-3)
        PT.append(1e-14 * float(h.max() - h.min()))  # runs to maxiter
    best = None
    for _ in range(reps + 1):  # the first run builds graphs and work lists
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        constrained_conjugate_gradients_batch(subs, hs, external_force=F, pentol=PT,
                                              forcetol=1e-16, maxiter=iters, precision=precision)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / iters
        best = dt if best is None else min(best, dt)
    return best


def tune_batch(sides=SIDES, precisions=("fp32", "fp64"), solves=512, iters=24, seed=0, log=None):
    """Measure and return a tuning table (see module docstring).  The
    objective is the iteration time of one batch of `solves` problems whose
    sides are drawn from `sides` (the batched workload's own mix): one pass of
    coordinate descent over the tile size of each sequence length, then the
    block threads.  The measurements are kept under "us_per_iteration"."""
    L = _lib.lib()
    shapes = _mix(sides, solves, seed)
    table = {"tiles": {}, "threads": {}, "us_per_iteration": {}, "device": _device_name(),
             "solves": solves, "iterations": iters, "sides": list(sides)}
    for prec in precisions:
        pi = _lib.PRECISIONS[prec]
        _lib.check(L.cm_tuning_set_batch_threads(pi, 256))
        for side in sides:
            _lib.check(L.cm_tuning_set_tiles(pi, side, 0))
        tiles, meas = {}, {}
        base = _batch_seconds(shapes, prec, iters, seed) * 1e6
        meas["default"] = round(base, 2)
        for side in sides:
            res = {}
            for elems in TILE_CANDIDATES[prec]:
                _lib.check(L.cm_tuning_set_tiles(pi, side, elems))
                res[elems] = _batch_seconds(shapes, prec, iters, seed) * 1e6
            pick = min(res, key=res.get)
            _lib.check(L.cm_tuning_set_tiles(pi, side, pick))
            tiles[str(side)] = pick
            meas[f"side{side}"] = {str(k): round(v, 2) for k, v in res.items()}
            if log:
                log(f"{prec} side {side}: {meas[f'side{side}']} -> {pick}")
        res = {}
        for threads in THREAD_CANDIDATES:
            _lib.check(L.cm_tuning_set_batch_threads(pi, threads))
            res[threads] = _batch_seconds(shapes, prec, iters, seed) * 1e6
        pick = min(res, key=res.get)
        _lib.check(L.cm_tuning_set_batch_threads(pi, pick))
        meas["threads"] = {str(k): round(v, 2) for k, v in res.items()}
        meas["tuned"] = round(res[pick], 2)
        if log:
            log(f"{prec} threads: {meas['threads']} -> {pick}; default {base:.1f} us")
        table["tiles"][prec] = tiles
        table["threads"][prec] = pick
        table["us_per_iteration"][prec] = meas
    return table


def _device_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return None


if __name__ == "__main__":
    import sys
    out = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_TABLE
    t = tune_batch(log=print)
    save(t, out)
    print("wrote", out)
