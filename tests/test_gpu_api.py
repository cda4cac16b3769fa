"""Entry points and failure paths of the device solver (GPU).

* cm_ccg_solve_host: the host-array entry point that a reference-side
  binding calls, through ctypes, against the oracle;
* the host-side time budget (timeout -> CM_ERR_TIMEOUT);
* a bounded device-side wait that runs out (the grid barrier of the
  one-launch offset bisection, made unreachable by phantom arrivals): every
  block gives up after its limit, the launch ends, and the next solve on
  the same device succeeds;
* NaN heights -> RuntimeError('nan encountered.')
  (ConstrainedConjugateGradients.py:491-492);
* pentol=None: the reference's default heuristic (:150-162);
* initial_forces (:211-215);
* FreeFFTElasticHalfSpace(check_boundaries=True) raising FreeBoundaryError
  through minimize_proxy (FFTElasticHalfSpace.py:1207-1283, Systems.py:610).
None of these faults, traps or hangs a GPU: the failures are made on the
host or end on a bounded wait.
"""
import ctypes

import numpy as np
import pytest

from oracle import contact_oracle as oc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def _rough(nb, seed=3, hurst=0.8, slope=0.1):
    return oc.self_affine(nb, (1.0, 1.0), hurst, slope, seed=seed)


def test_solve_host_entry_point_vs_oracle(cm):
    """cm_ccg_solve_host with numpy buffers (the binding INTEGRATION.md shows)."""
    from contactmechanics_b200 import _lib
    nb = (96, 80)
    h = np.ascontiguousarray(_rough(nb))
    F = 3e-3
    kw = dict(external_force=F, pentol=1e-11 * float(h.max() - h.min()), forcetol=1e-13)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    L = _lib.lib()
    P = _lib.CcgParams()
    P.precision, P.load_control, P.external_force = _lib.CM_FP64, 1, F
    P.pentol, P.forcetol, P.thermotol = kw["pentol"], kw["forcetol"], 1e-6
    P.mixfac, P.mixdecfac, P.minmixsteps, P.maxiter = 0.1, 0.95, 10, 100000
    x = np.empty(nb)
    jac = np.empty(nb)
    active = np.empty(nb, dtype=np.uint8)
    res = _lib.CcgResult()

    def p(a):
        return a.ctypes.data_as(ctypes.c_void_p)
    code = L.cm_ccg_solve_host(sub._plan.ptr, ctypes.byref(P), p(h), None, None, p(x), p(jac),
                               p(active), None, ctypes.byref(res))
    assert code == _lib.CM_OK, _lib.status_string(code)
    assert res.status == _lib.CM_SOLVE_CONVERGED
    ref = oc.constrained_conjugate_gradients(oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0)), h, **kw)
    np.testing.assert_allclose(x, ref["x"], rtol=0, atol=1e-10 * abs(ref["x"]).max())
    np.testing.assert_allclose(jac, ref["jac"], rtol=0, atol=1e-10 * abs(ref["jac"]).max())
    np.testing.assert_array_equal(active.astype(bool), ref["active_set"])
    assert res.nit == ref["nit"]
    np.testing.assert_allclose(res.offset, ref["offset"], rtol=1e-10)


def test_timeout_budget(cm):
    """A solve that cannot finish within its host-side budget returns
    CM_ERR_TIMEOUT (raised as CudaLibraryError) and leaves the plan usable."""
    from contactmechanics_b200 import _lib
    nb = (512, 512)
    h = _rough(nb, seed=9)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    kw = dict(external_force=5e-3, pentol=1e-13 * float(h.max() - h.min()), forcetol=1e-15)
    with pytest.raises(_lib.CudaLibraryError, match="time budget"):
        cm.constrained_conjugate_gradients(sub, h, timeout=1e-4, check_every=1, **kw)
    kw["pentol"] = 1e-10 * float(h.max() - h.min())
    res = cm.constrained_conjugate_gradients(sub, h, **kw)
    assert res.success


def test_device_wait_runs_out_and_context_stays_usable(cm):
    """The bounded grid barrier gives up when its arrivals never come."""
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    gave_up = ctypes.c_int(-1)
    # a barrier every block reaches completes
    assert L.cm_selftest_grid_barrier(8, 0, 1e5, ctypes.byref(gave_up)) == _lib.CM_OK
    assert gave_up.value == 0
    # phantom arrivals: the release count is never reached; every block gives
    # up after about 1 ms
    assert L.cm_selftest_grid_barrier(8, 8, 1e3, ctypes.byref(gave_up)) == _lib.CM_OK
    assert gave_up.value == 8
    torch.cuda.synchronize()
    nb = (64, 64)
    h = _rough(nb, seed=4, hurst=0.7, slope=0.2)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    kw = dict(external_force=4e-3, hardness=0.05 / (64 * 64), pentol=1e-11 * float(h.max() - h.min()),
              forcetol=1e-10)
    res = cm.constrained_conjugate_gradients(sub, h, **kw)
    ref = oc.constrained_conjugate_gradients(oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0)), h, **kw)
    assert res.success and ref["success"]
    np.testing.assert_allclose(res.x, ref["x"], rtol=0, atol=1e-10 * abs(ref["x"]).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_heights_raise(cm, precision):
    nb = (64, 64)
    h = _rough(nb)
    h[10, 20] = np.nan
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    with pytest.raises(RuntimeError, match="nan encountered"):
        cm.constrained_conjugate_gradients(sub, h, external_force=1e-3, pentol=1e-8,
                                           precision=precision)
    # the plan solves again afterwards
    h[10, 20] = 0.0
    assert cm.constrained_conjugate_gradients(sub, h, external_force=1e-3, pentol=1e-8,
                                              precision=precision).success


@pytest.mark.parametrize("kind", ["periodic", "free"])
def test_default_pentol_heuristic(cm, kind):
    """pentol=None: rms height / (10 mean(nb)) computed on the device."""
    nb = (64, 48)
    if kind == "free":
        h = oc.sphere(nb, (1.0, 1.0), 2.0)
        sub = cm.FreeFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
        o = oc.FreeSubstrate(nb, 1.0, (1.0, 1.0))
        kw = dict(offset=0.02)
    else:
        h = _rough(nb)
        sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
        o = oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0))
        kw = dict(external_force=2e-3)
    res = cm.constrained_conjugate_gradients(sub, h, forcetol=1e-12, **kw)
    ref = oc.constrained_conjugate_gradients(o, h, forcetol=1e-12, **kw)
    expected = oc.rms_height(h) / (10 * np.mean(h.shape))
    np.testing.assert_allclose(res.pentol, expected, rtol=1e-12)
    assert res.success and ref["success"]
    assert res.nit == ref["nit"]
    np.testing.assert_allclose(res.x, ref["x"], rtol=0, atol=1e-10 * abs(ref["x"]).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_initial_forces(cm, precision):
    """A warm start from forces (the force field of a nearby load)."""
    nb = (96, 96)
    h = _rough(nb, seed=12)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    o = oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0))
    kw = dict(pentol=1e-11 * float(h.max() - h.min()), forcetol=1e-13)
    first = oc.constrained_conjugate_gradients(o, h, external_force=2e-3, **kw)
    f0 = np.zeros(nb)
    f0[:, :] = -first["jac"]
    ref = oc.constrained_conjugate_gradients(o, h, external_force=3e-3, initial_forces=f0, **kw)
    res = cm.constrained_conjugate_gradients(sub, h, external_force=3e-3, initial_forces=f0,
                                             precision=precision, **kw)
    assert res.success and ref["success"]
    e = np.linalg.norm(res.x - ref["x"]) / np.linalg.norm(ref["x"])
    if precision == "fp64":
        assert res.nit == ref["nit"]
        assert e < 1e-10, e
    else:
        assert e < 1e-6, e


def test_check_boundaries_raises_through_minimize_proxy(cm):
    """A free contact that reaches the edge of the topography raises
    FreeBoundaryError from substrate.check() after the solve; one that stays
    inside does not."""
    from contactmechanics_b200.Topography import Topography
    nb = (64, 64)
    flat = np.zeros(nb)
    sys_ = cm.make_system(Topography(flat, (1.0, 1.0), periodic=False), substrate="free",
                          young=1.0, check_boundaries=True)
    with pytest.raises(cm.FreeFFTElasticHalfSpace.FreeBoundaryError):
        sys_.minimize_proxy(offset=1e-3, pentol=1e-10, forcetol=1e-12)
    sphere = oc.sphere(nb, (1.0, 1.0), 1.0)
    sys_ = cm.make_system(Topography(sphere, (1.0, 1.0), periodic=False), substrate="free",
                          young=1.0, check_boundaries=True)
    res = sys_.minimize_proxy(offset=1e-3, pentol=1e-10, forcetol=1e-12)
    assert res.success
