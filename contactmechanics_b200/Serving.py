"""Continuous-batching request loop for contact solves on one GPU.

Requests (one contact solve each: substrate geometry, heights, load or
offset, optional hardness) arrive at any time.  Between steps the loop
admits pending requests while free device memory allows, sets each admitted
solve up on a pooled plan (its heights, forces, search direction and
displacement stay on the device for the whole solve), advances every
in-flight solve by a few iterations in one batched launch sequence
(``cm_ccg_step``), hands mixed-precision solves over from their FP32 phase
to the FP64 refinement, and retires finished solves.  A solve's result does
not depend on which other solves share its steps.

Large requests (at least ``large_points`` domain points) skip the lockstep
batch: ``large_workers`` worker threads solve them with the single-solve
path (``constrained_conjugate_gradients``, which on domains with sides 2^k or
3 * 2^m runs the by-value passes of a CUDA graph on the plan's own stream), each one
request at a time, while the loop keeps stepping the small ones; the
single-solve passes are latency-bound, so two large solves on their own
streams overlap on the device.  Their results are those of
``constrained_conjugate_gradients`` for the same arguments.  Without
running threads, ``step`` solves a waiting large request itself.

Each request returns the same ``OptimizeResult`` as
``constrained_conjugate_gradients`` (numpy arrays), plus ``latency_s`` from
arrival to completion.
"""
import collections
import ctypes
import threading
import time

import numpy as np
import scipy.optimize as optim

from . import _lib
from .FFTElasticHalfSpace import FreeFFTElasticHalfSpace, PeriodicFFTElasticHalfSpace
from .Optimization.ConstrainedConjugateGradients import (_device_f64, _params,
                                                        constrained_conjugate_gradients)


def _torch():
    import torch
    return torch


def plan_bytes(kind, nb_grid_pts):
    """Device bytes one pooled plan holds (both precisions, tables, fields)."""
    nx, ny = nb_grid_pts
    if kind == "free":
        nx, ny = 2 * nx, 2 * ny
    nd, nt = nx * ny, nb_grid_pts[0] * nb_grid_pts[1]
    nh = nx * (ny // 2 + 8)
    fields = nd * (4 + 8) + nt * (4 + 8) * 4 + nt * 2
    spectra = nh * (8 + 16)
    tables = nh * (8 * 3 + 4 * 2)
    return fields + spectra + tables + (1 << 20)


class Request:
    """Handle of one submitted solve."""

    def __init__(self, rid, kind, nb_grid_pts, physical_sizes, young, heights, solver_kwargs,
                 arrival):
        self.id = rid
        self.kind = kind
        self.nb_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self.physical_sizes = tuple(float(s) for s in physical_sizes)
        self.young = float(young)
        self.heights = heights
        self.solver_kwargs = solver_kwargs
        self.arrival = arrival
        self.done_event = threading.Event()
        self.result_value = None
        self.error = None
        self.finished = None
        self._substrate = None
        self._h_dev = None
        self._u0_dev = None

    @property
    def key(self):
        return (self.kind, self.nb_grid_pts, self.physical_sizes, self.young)

    @property
    def latency_s(self):
        return None if self.finished is None else self.finished - self.arrival

    def result(self, timeout=None):
        if not self.done_event.wait(timeout):
            raise TimeoutError("request not finished")
        if self.error is not None:
            raise self.error
        return self.result_value


class ContactServer:
    """Admits, steps and retires contact solves (see module docstring).

    max_active       largest number of solves in flight
    iters_per_step   iterations every in-flight solve advances per step
    hbm_reserve      bytes of device memory kept free when admitting
    mem_info         callable returning (free, total) device bytes
                     (default: torch.cuda.mem_get_info)
    precision        "mixed", "fp64" or "fp32"
    large_points     requests with at least this many domain points are
                     solved by the single-solve path (None: every request
                     is batched); on the serving mix 2^18 (512^2) served
                     9.8 solves/s against 9.0 at 2^20
    large_workers    threads solving large requests concurrently
    """

    def __init__(self, max_active=512, iters_per_step=8, hbm_reserve=1 << 30, mem_info=None,
                 precision="mixed", large_points=1 << 18, large_workers=2):
        torch = _torch()
        self._L = _lib.lib()
        self._torch = torch
        ptr = ctypes.c_void_p()
        _lib.check(self._L.cm_stepper_create(None, ctypes.byref(ptr)))
        self._stepper = ptr
        self.max_active = max_active
        self.iters_per_step = iters_per_step
        self.hbm_reserve = hbm_reserve
        self.mem_info = mem_info or torch.cuda.mem_get_info
        self.precision = precision
        self._pending = collections.deque()
        self._large = collections.deque()
        self.large_points = large_points
        self._large_busy = 0       # large requests being solved
        self.large_workers = max(1, int(large_workers))
        self._workers = []
        self._active = []
        self._pool = collections.defaultdict(list)
        self._lock = threading.Lock()
        self._next_id = 0
        self._thread = None
        self._stop = threading.Event()
        self._wake = threading.Event()
        self._large_wake = threading.Event()
        self.completed = []
        self.steps = 0

    # ------------------------------------------------------------------ API
    def submit(self, kind, nb_grid_pts, physical_sizes, heights, young=1.0, arrival=None,
               **solver_kwargs):
        """Queue one solve; solver_kwargs as for constrained_conjugate_gradients
        (external_force or offset, hardness in force units, pentol, forcetol,
        thermotol, maxiter, initial_displacements)."""
        if kind not in ("periodic", "free"):
            raise ValueError("kind must be 'periodic' or 'free'")
        with self._lock:
            req = Request(self._next_id, kind, nb_grid_pts, physical_sizes, young, heights,
                          solver_kwargs, time.perf_counter() if arrival is None else arrival)
            self._next_id += 1
            if self._is_large(req):
                self._large.append(req)
            else:
                self._pending.append(req)
        self._wake.set()
        self._large_wake.set()
        return req

    def cancel(self, req):
        """Withdraw a request that has not been admitted yet."""
        with self._lock:
            try:
                self._pending.remove(req)
            except ValueError:
                try:
                    self._large.remove(req)
                except ValueError:
                    return False
        req.error = RuntimeError("cancelled")
        req.finished = time.perf_counter()
        req.done_event.set()
        return True

    @property
    def n_pending(self):
        return len(self._pending) + len(self._large)

    @property
    def n_active(self):
        return len(self._active)

    def step(self):
        """One scheduling round: admit, advance, hand over, retire.
        Returns the number of solves in flight after the round."""
        if not self._workers and self._large:
            self._solve_next_large()  # no worker threads: solve it here
        self._admit()
        if not self._active:
            return 0
        n = len(self._active)
        plans = (ctypes.c_void_p * n)(*[r._substrate._plan.ptr.value for r in self._active])
        done = (ctypes.c_int * n)()
        code = self._L.cm_ccg_step(self._stepper, n, plans, self.iters_per_step, done)
        _lib.check(code)
        self.steps += 1
        still = []
        for i, req in enumerate(self._active):
            if not done[i]:
                still.append(req)
                continue
            fin = ctypes.c_int()
            code = self._L.cm_ccg_handover(self._stepper, req._substrate._plan.ptr,
                                           ctypes.c_void_p(req._h_dev.data_ptr()), ctypes.byref(fin))
            if code != _lib.CM_OK:
                self._fail(req, code)
                continue
            if fin.value:
                self._finish(req)
            else:
                still.append(req)
        self._active = still
        return len(self._active)

    def run_until_idle(self, timeout=None):
        t0 = time.perf_counter()
        while self._pending or self._active or self._large or self._large_busy:
            if not self.step() and self._workers:
                time.sleep(0.0005)
            if timeout is not None and time.perf_counter() - t0 > timeout:
                raise TimeoutError("server did not drain")

    def start(self):
        """Drive step() from a background thread."""
        if self._thread is not None:
            return
        self._stop.clear()

        # each thread works on a stream of its own (torch streams do not wait
        # for other streams), so the loop's and the worker's small tensor
        # operations do not serialise against each other's solves
        device = self._torch.cuda.current_device()

        def loop():
            torch = self._torch
            torch.cuda.set_device(device)
            with torch.cuda.stream(torch.cuda.Stream()):
                while not self._stop.is_set():
                    if not self._pending and not self._active:
                        self._wake.wait(0.001)
                        self._wake.clear()
                        continue
                    self.step()

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

        def large_loop():
            torch = self._torch
            torch.cuda.set_device(device)
            with torch.cuda.stream(torch.cuda.Stream()):
                while not self._stop.is_set():
                    if not self._solve_next_large():
                        self._large_wake.wait(0.001)
                        self._large_wake.clear()

        for _ in range(self.large_workers):
            w = threading.Thread(target=large_loop, daemon=True)
            w.start()
            self._workers.append(w)

    def stop(self):
        if self._thread is None:
            return
        self._stop.set()
        self._wake.set()
        self._large_wake.set()
        self._thread.join()
        self._thread = None
        for w in self._workers:
            w.join()
        self._workers = []

    def close(self):
        self.stop()
        if self._stepper:
            self._L.cm_stepper_destroy(self._stepper)
            self._stepper = None

    # -------------------------------------------------------------- internals
    def _is_large(self, req):
        if self.large_points is None:
            return False
        f = 2 if req.kind == "free" else 1
        return f * f * int(np.prod(req.nb_grid_pts)) >= self.large_points

    def _solve_next_large(self):
        """Solve the oldest waiting large request with the single-solve path;
        False if there was none."""
        with self._lock:
            if not self._large:
                return False
            req = self._large.popleft()
            self._large_busy += 1
        try:
            with self._lock:
                sub = self._substrate(req)
            kw = dict(req.solver_kwargs)
            kw.setdefault("precision", self.precision)
            try:
                r = constrained_conjugate_gradients(sub, req.heights, **kw)
                for key in ("x", "jac", "active_set", "plastic"):
                    v = getattr(r, key, None)
                    if v is not None and hasattr(v, "cpu"):
                        setattr(r, key, v.cpu().numpy())
                req.result_value = r
                req.finished = time.perf_counter()
                r.latency_s = req.latency_s
                self.completed.append(req)
            except Exception as exc:  # invalid request: report it, keep serving
                req.error = exc
                req.finished = time.perf_counter()
            finally:
                with self._lock:
                    self._pool[req.key].append(sub)
            req.done_event.set()
        finally:
            with self._lock:
                self._large_busy -= 1
        return True

    def _substrate(self, req):
        pool = self._pool[req.key]
        if pool:
            return pool.pop()
        if req.kind == "free":
            return FreeFFTElasticHalfSpace(req.nb_grid_pts, req.young, req.physical_sizes)
        return PeriodicFFTElasticHalfSpace(req.nb_grid_pts, req.young, req.physical_sizes)

    def _admit(self):
        with self._lock:
            if not self._pending:
                return
            free = int(self.mem_info()[0])
            keep = collections.deque()
            while self._pending:
                req = self._pending.popleft()
                need = 0 if self._pool[req.key] else plan_bytes(req.kind, req.nb_grid_pts)
                if len(self._active) >= self.max_active or free - need < self.hbm_reserve:
                    keep.append(req)
                    continue
                free -= need
                try:
                    self._begin(req)
                    self._active.append(req)
                except Exception as exc:  # invalid request: report it, keep serving
                    req.error = exc
                    req.finished = time.perf_counter()
                    req.done_event.set()
            self._pending = keep

    def _begin(self, req):
        kw = dict(req.solver_kwargs)
        sub = self._substrate(req)
        req._substrate = sub
        req._h_dev = _device_f64(req.heights, sub.nb_grid_pts, role="h")
        u0 = kw.pop("initial_displacements", None)
        req._u0_dev = (_device_f64(u0, sub.nb_domain_grid_pts, role="u0")
                       if u0 is not None else None)
        P = _params(self.precision, kw.get("external_force"), kw.get("offset"), kw.get("hardness"),
                    kw.get("pentol"), kw.get("forcetol", 1e-5), kw.get("thermotol", 1e-6),
                    kw.get("mixfac", 0.1), kw.get("mixdecfac", 0.95), kw.get("minmixsteps", 10),
                    kw.get("maxiter", 100000))
        if P.has_hardness and not P.hardness > 0:
            raise ValueError("hardness must be positive")
        req._params = P
        self._torch.cuda.current_stream().synchronize()
        code = self._L.cm_ccg_begin(self._stepper, sub._plan.ptr, ctypes.byref(P),
                                    ctypes.c_void_p(req._h_dev.data_ptr()),
                                    ctypes.c_void_p(req._u0_dev.data_ptr()) if req._u0_dev is not None
                                    else None, None)
        if code != _lib.CM_OK:
            self._pool[req.key].append(sub)
            raise _lib.CudaLibraryError(_lib.status_string(code))

    def _release(self, req):
        if req._substrate is not None:
            self._pool[req.key].append(req._substrate)
            req._substrate = None
        req._h_dev = req._u0_dev = None

    def _fail(self, req, code):
        msgs = {_lib.CM_ERR_NAN: RuntimeError("nan encountered."),
                _lib.CM_ERR_BISECT: ValueError("f(a) and f(b) must have different signs"),
                _lib.CM_ERR_BISECT_CONV: RuntimeError("Failed to converge after 100 iterations")}
        req.error = msgs.get(code, _lib.CudaLibraryError(_lib.status_string(code)))
        req.finished = time.perf_counter()
        self._release(req)
        req.done_event.set()

    def _finish(self, req):
        torch = self._torch
        sub = req._substrate
        nb, dom = tuple(sub.nb_grid_pts), tuple(sub.nb_domain_grid_pts)
        x = torch.empty(dom, dtype=torch.float64, device="cuda")
        jac = torch.empty(nb, dtype=torch.float64, device="cuda")
        act = torch.empty(nb, dtype=torch.uint8, device="cuda")
        has_h = req._params.has_hardness
        pl = torch.empty(nb, dtype=torch.uint8, device="cuda") if has_h else None
        res = _lib.CcgResult()
        code = self._L.cm_ccg_end(self._stepper, sub._plan.ptr, ctypes.c_void_p(x.data_ptr()),
                                  ctypes.c_void_p(jac.data_ptr()), ctypes.c_void_p(act.data_ptr()),
                                  ctypes.c_void_p(pl.data_ptr()) if pl is not None else None,
                                  ctypes.byref(res))
        if code != _lib.CM_OK:
            self._fail(req, code)
            return
        maxiter = req.solver_kwargs.get("maxiter", 100000)
        r = optim.OptimizeResult()
        r.nit, r.nfev, r.nit_fp32 = res.nit, res.nfev, res.nit_fp32
        r.success = res.status == _lib.CM_SOLVE_CONVERGED
        r.message = "Polonsky converged" if r.success else "Reached maxiter = {}".format(maxiter)
        r.maxcv = {"max_pen": res.max_pen, "max_pres": res.max_pres}
        r.offset, r.fun, r.pentol = res.offset, res.fun, res.pentol_used
        act_dom = np.zeros(dom, dtype=bool)
        act_dom[:nb[0], :nb[1]] = act.cpu().numpy().astype(bool)
        r.x, r.jac, r.active_set = x.cpu().numpy(), jac.cpu().numpy(), act_dom
        if pl is not None and r.success:
            r.plastic = pl.cpu().numpy().astype(bool)
        req.result_value = r
        req.finished = time.perf_counter()
        r.latency_s = req.latency_s
        self._release(req)
        self.completed.append(req)
        req.done_event.set()
