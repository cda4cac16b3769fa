"""ctypes binding of libcm_b200.so (the C ABI declared in include/cm_b200.h).

The shared library is built in-tree (``contactmechanics_b200/lib``) by
``contactmechanics_b200.build``.  There is no CPU fallback: if the library
or a CUDA device is missing, :func:`lib` raises.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcm_b200.so")

CM_OK = 0
CM_ERR_ARG = 1
CM_ERR_SHAPE = 2
CM_ERR_SIZE = 3
CM_ERR_CUDA = 4
CM_ERR_OOM = 5
CM_ERR_NAN = 6
CM_ERR_BISECT = 7
CM_ERR_BISECT_CONV = 8
CM_ERR_TIMEOUT = 9
CM_ERR_STOPPED = 10

CM_PERIODIC = 0
CM_FREE = 1
CM_SEMI = 2
CM_FP64 = 0
CM_FP32 = 1
CM_MIXED = 2
CM_Q0_DEFAULT = 0
CM_Q0_ZERO = 1
CM_Q0_VALUE = 2
CM_OP_DISP = 0
CM_OP_FORCE = 1
CM_SOLVE_CONVERGED = 1
CM_SOLVE_MAXITER = 2
CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream

PRECISIONS = {"fp64": CM_FP64, "fp32": CM_FP32, "mixed": CM_MIXED}


class PlanDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("dim", ctypes.c_int),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("sx", ctypes.c_double), ("sy", ctypes.c_double),
                ("young", ctypes.c_double), ("poisson", ctypes.c_double),
                ("q0_mode", ctypes.c_int), ("stiffness_q0", ctypes.c_double),
                ("thickness", ctypes.c_double), ("periodic_x", ctypes.c_int),
                ("periodic_y", ctypes.c_int), ("n_images", ctypes.c_int)]


class Iteration(ctypes.Structure):
    """cm_iteration: one CCG iteration as the per-iteration observer sees it."""
    _fields_ = [("it", ctypes.c_int), ("precision", ctypes.c_int), ("mode", ctypes.c_int),
                ("done", ctypes.c_int), ("area", ctypes.c_longlong),
                ("cg_area", ctypes.c_longlong), ("plastic_area", ctypes.c_longlong),
                ("nc_count", ctypes.c_longlong),
                ("rms_pen", ctypes.c_double), ("max_pen", ctypes.c_double),
                ("max_pres", ctypes.c_double), ("pad_pres", ctypes.c_double),
                ("maxdu", ctypes.c_double), ("total_force", ctypes.c_double),
                ("offset", ctypes.c_double), ("tau", ctypes.c_double),
                ("mixfac", ctypes.c_double), ("pentol", ctypes.c_double),
                ("forcetol", ctypes.c_double), ("forces", ctypes.c_void_p)]


ITERATION_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(Iteration))


class CcgParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("load_control", ctypes.c_int),
                ("external_force", ctypes.c_double), ("offset", ctypes.c_double),
                ("has_hardness", ctypes.c_int), ("hardness", ctypes.c_double),
                ("pentol", ctypes.c_double), ("forcetol", ctypes.c_double),
                ("thermotol", ctypes.c_double), ("mixfac", ctypes.c_double),
                ("mixdecfac", ctypes.c_double), ("minmixsteps", ctypes.c_int),
                ("maxiter", ctypes.c_int), ("check_every", ctypes.c_int),
                ("fp32_pentol_rel", ctypes.c_double), ("timeout_s", ctypes.c_double),
                ("on_iteration", ITERATION_FN), ("user", ctypes.c_void_p),
                ("iteration_forces", ctypes.c_void_p)]


class CcgResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("nit", ctypes.c_int), ("nfev", ctypes.c_int),
                ("nit_fp32", ctypes.c_int), ("last_step_mix", ctypes.c_int),
                ("offset", ctypes.c_double), ("fun", ctypes.c_double),
                ("rms_pen", ctypes.c_double), ("max_pen", ctypes.c_double),
                ("max_pres", ctypes.c_double), ("pad_pres", ctypes.c_double),
                ("maxdu", ctypes.c_double), ("total_force", ctypes.c_double),
                ("pentol_used", ctypes.c_double),
                ("area", ctypes.c_longlong), ("cg_area", ctypes.c_longlong),
                ("plastic_area", ctypes.c_longlong), ("ms_fp32", ctypes.c_double),
                ("ms_fp64", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("polls", ctypes.c_int)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
# exported symbol -> (restype, argtypes); every symbol of include/cm_b200.h
SIGNATURES = {
    "cm_status_string": (ctypes.c_char_p, [_i]),
    "cm_version": (ctypes.c_char_p, []),
    "cm_plan_create": (_i, [ctypes.POINTER(PlanDesc), _vp, ctypes.POINTER(_vp)]),
    "cm_plan_destroy": (_i, [_vp]),
    "cm_plan_shape": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "cm_plan_engine": (_i, [_vp, _i, ctypes.POINTER(_i)]),
    "cm_plan_greens_host": (_i, [_vp, _vp]),
    "cm_apply": (_i, [_vp, _i, _i, _vp, _i, _i, _i, _vp, _i, _i, _i, _vp]),
    "cm_ccg_solve": (_i, [_vp, ctypes.POINTER(CcgParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                          ctypes.POINTER(CcgResult)]),
    "cm_ccg_solve_host": (_i, [_vp, ctypes.POINTER(CcgParams), _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, ctypes.POINTER(CcgResult)]),
    "cm_ccg_solve_batch": (_i, [_i, _vp, ctypes.POINTER(CcgParams), _vp, _vp, _vp, _vp, _vp, _vp,
                                ctypes.POINTER(CcgResult), _vp]),
    "cm_stepper_create": (_i, [_vp, ctypes.POINTER(_vp)]),
    "cm_stepper_destroy": (_i, [_vp]),
    "cm_ccg_begin": (_i, [_vp, _vp, ctypes.POINTER(CcgParams), _vp, _vp, _vp]),
    "cm_ccg_step": (_i, [_vp, _i, _vp, _i, ctypes.POINTER(_i)]),
    "cm_ccg_handover": (_i, [_vp, _vp, _vp, ctypes.POINTER(_i)]),
    "cm_ccg_end": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(CcgResult)]),
    "cm_launch_count": (ctypes.c_ulonglong, []),
    "cm_apply_periodic_noalloc": (_i, [_i, _i, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _i, _vp, _vp, _vp]),
    "cm_selftest_grid_barrier": (_i, [_i, _i, ctypes.c_double, ctypes.POINTER(_i)]),
    "cm_tuning_set_tiles": (_i, [_i, _i, _i]),
    "cm_tuning_set_batch_threads": (_i, [_i, _i]),
    "cm_tuning_get": (_i, [_i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "cm_tuning_set_batch_persistent": (_i, [_i]),
    "cm_fft_forward": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp]),
    "cm_kspace_apply": (_i, [_vp, _i, ctypes.c_double, _vp, _vp, _vp]),
    "cm_kspace_dot": (_i, [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double), _vp]),
    "cm_ccg_profile": (_i, [_vp, ctypes.POINTER(CcgParams), _vp, _i,
                            ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_i),
                            ctypes.POINTER(ctypes.c_char_p)]),
}

_lock = threading.Lock()
_lib = None


class CudaLibraryError(RuntimeError):
    """Raised when the CUDA library or device is unavailable or fails."""


def load_library(path=LIB_PATH):
    """Load the shared library and declare every exported signature.

    Does not touch the GPU, so it works on a machine without one."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise CudaLibraryError(
                f"{path} is missing; build it with `python -m contactmechanics_b200.build`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def lib():
    """The loaded library; raises if no CUDA device is usable."""
    import torch
    if not torch.cuda.is_available():
        raise CudaLibraryError("contactmechanics_b200 needs a CUDA device (B200); none is available")
    return load_library()


def status_string(code):
    return load_library().cm_status_string(code).decode()


def check(code, error_cls=CudaLibraryError):
    if code != CM_OK:
        raise error_cls(status_string(code))
