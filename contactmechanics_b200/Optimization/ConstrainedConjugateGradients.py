"""Polonsky-Keer constrained conjugate gradients on the B200.

Drop-in for ``constrained_conjugate_gradients`` of
ContactMechanics/Optimization/ConstrainedConjugateGradients.py (v1.8.3):
same arguments, same ``OptimizeResult`` fields, same exceptions.  The whole
iteration -- both operator applications, every masked reduction, the step
length, the projection onto [0, hardness], the load constraint, the
mixing step with its offset bisection and the convergence test -- runs on
the device (``cm_ccg_solve`` of libcm_b200.so); the host only polls a
convergence flag every few iterations.

``callback(it, f_r, d)`` and the logger's per-iteration rows follow the
reference (:436-489): every iteration that does not converge is reported
(the loop then polls the device after each iteration instead of every few);
``f_r`` is the iteration's force field on the domain (a CUDA tensor when
the heights were one, else a numpy array).  In a mixed-precision solve the
FP64 refinement continues the FP32 phase's iteration count.

Differences that follow from keeping the loop on the device:
* masked (``np.ma``) heights and MPI domain decomposition are not supported;
* a scalar ``hardness`` must be positive (the reference fails later, inside
  its bisection, for ``hardness == 0``).

Extra keyword ``precision``: "fp64" (default; reference arithmetic),
"mixed" (FP32 fields and FFTs with FP64 reductions, then FP64 refinement
iterations warm-started from the FP32 forces) or "fp32".
"""
import ctypes
import threading

import numpy as np
import scipy.optimize as optim

from .. import _lib
from ..Tools.Logger import quiet


def _torch():
    import torch
    return torch


class _Staging(threading.local):
    """Pinned host buffers of this thread, one per role (grown on demand), each
    with the event of the last copy through it."""

    def __init__(self):
        self.bufs = {}


_STAGING = _Staging()


def _pinned(role, n, dtype):
    torch = _torch()
    ent = _STAGING.bufs.get((role, dtype))
    if ent is None or ent[0].numel() < n:
        ent = [torch.empty(max(n, 1), dtype=dtype, pin_memory=True), None]
        _STAGING.bufs[(role, dtype)] = ent
    if ent[1] is not None:
        ent[1].synchronize()  # the previous copy through this buffer has finished
        ent[1] = None
    return ent


def _device_f64(a, shape=None, role="in"):
    """A float64 device copy of `a`; host arrays travel through a pinned buffer."""
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=torch.float64).contiguous()
    else:
        arr = np.asarray(a, dtype=np.float64)
        src = (torch.from_numpy(arr) if arr.flags.c_contiguous and arr.flags.writeable
               else None)
        if src is not None and src.is_pinned():
            # already page-locked (e.g. an earlier result of this module): one
            # DMA, complete before any solve starts (the callers synchronise
            # the stream before handing the inputs to the library)
            t = src.to("cuda", non_blocking=True)
        else:
            ent = _pinned(role, arr.size, torch.float64)
            host = ent[0][:arr.size]
            np.copyto(host.numpy().reshape(arr.shape), arr)
            t = host.to("cuda", non_blocking=True).reshape(arr.shape)
            ev = torch.cuda.Event()
            ev.record()
            ent[1] = ev
    if shape is not None:
        t = t.reshape(shape)
    return t


def _host_arrays(named):
    """numpy results of device tensors [(role, tensor), ...]: each is copied
    once, straight into page-locked host memory that the returned array
    views (torch's caching host allocator hands the memory out again once
    the array is released), so no host-side copy follows the transfer."""
    torch = _torch()
    hosts = []
    for role, t in named:
        h = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        hosts.append(h)
    torch.cuda.current_stream().synchronize()
    return [h.numpy() for h in hosts]


def constrained_conjugate_gradients(substrate, topography, hardness=None, external_force=None,
                                    offset=None, initial_displacements=None,
                                    initial_forces=None, pentol=None, forcetol=1e-5,
                                    thermotol=1e-6, mixfac=0.1, mixdecfac=0.95,
                                    minmixsteps=10, maxiter=100000, logger=quiet,
                                    callback=None, verbose=False, precision="fp64",
                                    check_every=None, timeout=None):
    """Equilibrium of an elastic half-space against a rigid topography
    (ConstrainedConjugateGradients.py:47-509).

    Returns a ``scipy.optimize.OptimizeResult`` with ``x`` (displacements on
    the full domain), ``jac`` (forces on the topography, positive in
    compression), ``active_set``, ``offset``, ``fun`` (elastic energy),
    ``success``, ``message``, ``nit``, ``nfev``, ``maxcv`` and, with a
    hardness, ``plastic``.
    """
    torch = _torch()
    plan = getattr(substrate, "_plan", None)
    if plan is None:
        raise ValueError("substrate must be a contactmechanics_b200 half-space")
    if not hasattr(topography, "nb_grid_pts"):
        heights = topography
    else:
        heights = topography.heights()
    if np.ma.isMaskedArray(heights):
        raise NotImplementedError("masked topographies are not supported on the device path")
    if substrate.dim not in (1, 2):
        raise Exception(
            f"Constrained conjugate gradient currently only implemented for 1 or 2 dimensions "
            f"(Your substrate has {substrate.dim}.).")
    as_torch = isinstance(heights, torch.Tensor) and heights.is_cuda
    nb = tuple(substrate.nb_grid_pts)
    tshape = nb if substrate.dim == 2 else (nb[0], 1)
    dom = tuple(substrate.nb_domain_grid_pts)
    dshape = dom if substrate.dim == 2 else (dom[0], 1)
    if tuple(heights.shape) != nb:
        raise ValueError("topography shape {} does not match the substrate's nb_grid_pts {}"
                         .format(tuple(heights.shape), nb))
    if hardness is not None:
        h_arr = np.asarray(hardness.cpu() if isinstance(hardness, torch.Tensor) else hardness)
        if h_arr.size != 1:
            raise ValueError("The truth value of an array with more than one element is "
                             "ambiguous. Use a.any() or a.all()")
        hardness = float(h_arr)
        if not hardness > 0:
            raise ValueError("hardness must be positive")
    if precision not in _lib.PRECISIONS:
        raise ValueError("precision must be one of {}".format(sorted(_lib.PRECISIONS)))

    h_dev = _device_f64(heights, tshape, role="h")
    u0 = (_device_f64(initial_displacements, dshape, role="u0")
          if initial_displacements is not None else None)
    f0 = _device_f64(initial_forces, dshape, role="f0") if initial_forces is not None else None
    x = torch.empty(dshape, dtype=torch.float64, device="cuda")
    jac = torch.empty(tshape, dtype=torch.float64, device="cuda")
    active = torch.empty(tshape, dtype=torch.uint8, device="cuda")
    plastic = torch.empty(tshape, dtype=torch.uint8, device="cuda") if hardness is not None else None

    P = _lib.CcgParams()
    P.precision = _lib.PRECISIONS[precision]
    P.load_control = int(external_force is not None)
    P.external_force = float(external_force) if external_force is not None else 0.0
    P.offset = float(offset) if offset is not None else 0.0
    P.has_hardness = int(hardness is not None)
    P.hardness = hardness if hardness is not None else 0.0
    P.pentol = float(pentol) if pentol is not None else -1.0
    P.forcetol = float(forcetol)
    P.thermotol = float(thermotol)
    P.mixfac = float(mixfac)
    P.mixdecfac = float(mixdecfac)
    P.minmixsteps = int(minmixsteps)
    P.maxiter = int(maxiter)
    P.check_every = int(check_every) if check_every else 0
    P.timeout_s = float(timeout) if timeout else 0.0
    res = _lib.CcgResult()
    errors = []
    observer = None
    if callback is not None or logger is not quiet:
        fbuf = torch.empty(dshape, dtype=torch.float64, device="cuda")
        observer = _observer(callback, logger, verbose, hardness is not None, maxiter, fbuf, dom,
                             as_torch, float(np.prod(tshape)), forcetol, errors)
        P.on_iteration = observer
        P.iteration_forces = fbuf.data_ptr()

    def ptr(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    torch.cuda.current_stream().synchronize()
    code = plan._L.cm_ccg_solve(plan.ptr, ctypes.byref(P), ptr(h_dev), ptr(u0), ptr(f0),
                                ptr(x), ptr(jac), ptr(active), ptr(plastic), ctypes.byref(res))
    if errors:
        raise errors[0]  # the callback's own exception stopped the solve
    if code == _lib.CM_ERR_NAN:
        raise RuntimeError("nan encountered.")
    if code == _lib.CM_ERR_BISECT:
        raise ValueError("f(a) and f(b) must have different signs")
    if code == _lib.CM_ERR_BISECT_CONV:
        raise RuntimeError("Failed to converge after 100 iterations")
    _lib.check(code)

    result = optim.OptimizeResult()
    result.nit = res.nit
    result.nfev = res.nfev
    result.nit_fp32 = res.nit_fp32
    result.success = res.status == _lib.CM_SOLVE_CONVERGED
    result.message = ("Polonsky converged" if result.success
                      else "Reached maxiter = {}".format(maxiter))
    result.maxcv = {"max_pen": res.max_pen, "max_pres": res.max_pres}
    result.offset = res.offset
    result.fun = res.fun
    result.pentol = res.pentol_used
    result.timing = {"ms_fp32": res.ms_fp32, "ms_fp64": res.ms_fp64, "ms_total": res.ms_total,
                     "polls": res.polls}

    # active set over the full domain (False on the padding)
    act_dom = torch.zeros(dshape, dtype=torch.bool, device="cuda")
    act_dom[:tshape[0], :tshape[1]] = active.bool()
    if substrate.dim == 1:
        x, jac, act_dom = x.reshape(dom), jac.reshape(nb), act_dom.reshape(dom)
        if plastic is not None:
            plastic = plastic.reshape(nb)
    if as_torch:
        result.x, result.jac, result.active_set = x, jac, act_dom
        if plastic is not None and result.success:
            result.plastic = plastic.bool()
    else:
        named = [("x", x), ("jac", jac), ("active", act_dom)]
        if plastic is not None and result.success:
            named.append(("plastic", plastic.bool()))
        arrays = _host_arrays(named)
        result.x, result.jac, result.active_set = arrays[:3]
        if len(arrays) > 3:
            result.plastic = arrays[3]

    log_headers = ["status", "it", "area", "cg area", "total force", "offset"]
    log_values = ["CONVERGED" if result.success else "NOT CONVERGED", res.nit, res.area,
                  res.cg_area, res.total_force, res.offset]
    if verbose:
        log_headers += ["rms pen.", "max. pen.", "max. force", "max. pad force", "max. du"]
        log_values += [res.rms_pen, res.max_pen, res.max_pres, res.pad_pres, res.maxdu]
    logger.pr(f"maxiter = {maxiter}")
    logger.pr(f"pentol = {res.pentol_used}")
    logger.st(log_headers, log_values, force_print=True)
    return result


_MODE_STR = {1: "sd", 2: "cg", 3: "mix"}


def _observer(callback, logger, verbose, plastic, maxiter, fbuf, dom, as_torch, n_surface,
              forcetol, errors):
    """The per-iteration observer handed to cm_ccg_solve: the reference's
    logger row and callback(it, f_r, d) (ConstrainedConjugateGradients.py
    :436-489) from the iteration's state and forces.  An exception stops the
    solve and is re-raised by the caller."""
    def on_iteration(user, info_p):
        try:
            i = info_p.contents
            if logger is not quiet and i.it < maxiter:
                hdr = ["status", "it", "area", "frac. area", "cg area", "total force", "offset"]
                val = [_MODE_STR.get(i.mode, "sd"), i.it, i.area, i.area / n_surface, i.cg_area,
                       i.total_force, i.offset]
                if plastic:
                    hdr += ["plast. area", "frac.plast. area"]
                    val += [i.plastic_area, i.plastic_area / n_surface]
                if verbose:
                    hdr += ["rms pen.", "max. pen.", "max. force", "max. pad force", "max. du",
                            "CG area", "frac. CG area", "sum(nc_r)"]
                    val += [i.rms_pen, i.max_pen, i.max_pres, i.pad_pres, i.maxdu, i.cg_area,
                            i.cg_area / n_surface, i.nc_count]
                    hdr += ["mixfac"] if i.mode == 3 else ["tau"]
                    val += [i.mixfac] if i.mode == 3 else [i.tau]
                logger.st(hdr, val)
            if callback is not None:
                f_r = fbuf.reshape(dom)
                if not as_torch:
                    f_r = f_r.cpu().numpy()
                d = dict(area=int(i.area), fractional_area=i.area / n_surface,
                         rms_penetration=i.rms_pen, max_penetration=i.max_pen,
                         max_pressure=i.max_pres, pad_pressure=i.pad_pres,
                         penetration_tol=i.pentol, pressure_tol=forcetol)
                callback(i.it, f_r, d)
            return 0
        except BaseException as e:  # cannot cross the C frames: stop and re-raise
            errors.append(e)
            return 1
    return _lib.ITERATION_FN(on_iteration)


def _params(precision, external_force, offset, hardness, pentol, forcetol, thermotol, mixfac,
            mixdecfac, minmixsteps, maxiter, timeout=None):
    P = _lib.CcgParams()
    P.precision = _lib.PRECISIONS[precision]
    P.load_control = int(external_force is not None)
    P.external_force = float(external_force) if external_force is not None else 0.0
    P.offset = float(offset) if offset is not None else 0.0
    P.has_hardness = int(hardness is not None)
    P.hardness = float(hardness) if hardness is not None else 0.0
    P.pentol = float(pentol) if pentol is not None else -1.0
    P.forcetol = float(forcetol)
    P.thermotol = float(thermotol)
    P.mixfac = float(mixfac)
    P.mixdecfac = float(mixdecfac)
    P.minmixsteps = int(minmixsteps)
    P.maxiter = int(maxiter)
    P.timeout_s = float(timeout) if timeout else 0.0
    return P


def _per_solve(value, n, name):
    if value is None or np.isscalar(value):
        return [value] * n
    value = list(value)
    if len(value) != n:
        raise ValueError(f"{name} needs one entry per solve")
    return value


def constrained_conjugate_gradients_batch(substrates, topographies, hardness=None,
                                          external_force=None, offset=None,
                                          initial_displacements=None, pentol=None,
                                          forcetol=1e-5, thermotol=1e-6, mixfac=0.1,
                                          mixdecfac=0.95, minmixsteps=10, maxiter=100000,
                                          precision="fp64", timeout=None):
    """Solve several independent contact problems together.

    ``substrates`` and ``topographies`` are sequences of equal length (one
    substrate per solve; grid sizes may differ).  ``hardness``,
    ``external_force``, ``offset``, ``initial_displacements``, ``pentol``
    and ``forcetol`` are scalars applied to every solve or sequences with one
    entry per solve.  Every solve keeps the semantics of
    :func:`constrained_conjugate_gradients`; all solves advance together on the
    device (``cm_ccg_solve_batch``).  Returns a list of ``OptimizeResult``.
    """
    torch = _torch()
    n = len(substrates)
    if n == 0 or len(topographies) != n:
        raise ValueError("need one topography per substrate")
    if precision not in _lib.PRECISIONS:
        raise ValueError("precision must be one of {}".format(sorted(_lib.PRECISIONS)))
    H = _per_solve(hardness, n, "hardness")
    F = _per_solve(external_force, n, "external_force")
    O = _per_solve(offset, n, "offset")
    U0 = (_per_solve(initial_displacements, n, "initial_displacements")
          if initial_displacements is not None and not hasattr(initial_displacements, "shape")
          else [initial_displacements] * n)
    PT = _per_solve(pentol, n, "pentol")
    FT = _per_solve(forcetol, n, "forcetol")
    plans, params, keep = [], [], []
    hs, u0s, xs, jacs, acts, pls = [], [], [], [], [], []
    as_torch = []
    for i in range(n):
        sub, topo = substrates[i], topographies[i]
        if getattr(sub, "_plan", None) is None or sub.dim != 2:
            raise ValueError("batch solves need 2D contactmechanics_b200 half-spaces")
        heights = topo.heights() if hasattr(topo, "nb_grid_pts") else topo
        if tuple(heights.shape) != tuple(sub.nb_grid_pts):
            raise ValueError("topography shape does not match its substrate")
        if H[i] is not None and not float(H[i]) > 0:
            raise ValueError("hardness must be positive")
        as_torch.append(isinstance(heights, torch.Tensor) and heights.is_cuda)
        dom = tuple(sub.nb_domain_grid_pts)
        h = _device_f64(heights)
        u0 = _device_f64(U0[i], dom) if U0[i] is not None else None
        x = torch.empty(dom, dtype=torch.float64, device="cuda")
        jac = torch.empty(tuple(sub.nb_grid_pts), dtype=torch.float64, device="cuda")
        act = torch.empty(tuple(sub.nb_grid_pts), dtype=torch.uint8, device="cuda")
        pl = torch.empty(tuple(sub.nb_grid_pts), dtype=torch.uint8, device="cuda") if H[i] is not None else None
        keep += [h, u0, x, jac, act, pl]
        hs.append(h); u0s.append(u0); xs.append(x); jacs.append(jac); acts.append(act); pls.append(pl)
        plans.append(sub._plan.ptr)
        params.append(_params(precision, F[i], O[i], H[i], PT[i], FT[i], thermotol, mixfac,
                              mixdecfac, minmixsteps, maxiter, timeout))

    def arr(ts):
        return (ctypes.c_void_p * n)(*[t.data_ptr() if t is not None else None for t in ts])

    plan_arr = (ctypes.c_void_p * n)(*[p.value for p in plans])
    par_arr = (_lib.CcgParams * n)(*params)
    res_arr = (_lib.CcgResult * n)()
    torch.cuda.current_stream().synchronize()
    L = substrates[0]._plan._L
    code = L.cm_ccg_solve_batch(n, plan_arr, par_arr, arr(hs), arr(u0s), arr(xs), arr(jacs),
                                arr(acts), arr(pls), res_arr, None)
    if code == _lib.CM_ERR_NAN:
        raise RuntimeError("nan encountered.")
    if code == _lib.CM_ERR_BISECT:
        raise ValueError("f(a) and f(b) must have different signs")
    if code == _lib.CM_ERR_BISECT_CONV:
        raise RuntimeError("Failed to converge after 100 iterations")
    _lib.check(code)
    out = []
    for i in range(n):
        r = res_arr[i]
        result = optim.OptimizeResult()
        result.nit, result.nfev, result.nit_fp32 = r.nit, r.nfev, r.nit_fp32
        result.success = r.status == _lib.CM_SOLVE_CONVERGED
        result.message = ("Polonsky converged" if result.success
                          else "Reached maxiter = {}".format(maxiter))
        result.maxcv = {"max_pen": r.max_pen, "max_pres": r.max_pres}
        result.offset, result.fun, result.pentol = r.offset, r.fun, r.pentol_used
        result.timing = {"ms_fp32": r.ms_fp32, "ms_fp64": r.ms_fp64, "ms_total": r.ms_total,
                         "polls": r.polls}
        sub = substrates[i]
        nb, dom = tuple(sub.nb_grid_pts), tuple(sub.nb_domain_grid_pts)
        act = acts[i].view(torch.bool)  # the library writes 0/1 bytes
        if dom == nb:
            act_dom = act
        else:
            act_dom = torch.zeros(dom, dtype=torch.bool, device="cuda")
            act_dom[:nb[0], :nb[1]] = act
        if as_torch[i]:
            result.x, result.jac, result.active_set = xs[i], jacs[i], act_dom
            if pls[i] is not None and result.success:
                result.plastic = pls[i].view(torch.bool)
        else:
            result.x, result.jac = xs[i].cpu().numpy(), jacs[i].cpu().numpy()
            result.active_set = act_dom.cpu().numpy()
            if pls[i] is not None and result.success:
                result.plastic = pls[i].view(torch.bool).cpu().numpy()
        out.append(result)
    return out
