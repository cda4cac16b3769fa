"""Domain sides 3 * 2^m (96 .. 6144; FP64 at 6144 on one transform buffer
with staged twiddles) on the register-resident passes: the
operator (FFTElasticHalfSpace.py:573-611, free :1141-1197) and the CCG solve
(ConstrainedConjugateGradients.py:200-489) against the oracle, with the same
tolerances as the power-of-two sizes, plus a check that these plans really
take those passes (cm_plan_engine) and give the same bits twice.
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


def _engine(sub, precision):
    from contactmechanics_b200 import _lib
    e = ctypes.c_int(-1)
    _lib.check(sub._plan._L.cm_plan_engine(sub._plan.ptr, _lib.PRECISIONS[precision],
                                           ctypes.byref(e)))
    return e.value


def _rel(u, v):
    return np.linalg.norm(u - v) / np.linalg.norm(v)


@pytest.mark.parametrize("nx, ny", [(96, 96), (192, 384), (96, 128), (256, 768), (1536, 1536),
                                     (3072, 64), (6144, 96)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_periodic_operator_vs_oracle(cm, nx, ny, precision):
    """Square, rectangular and mixed (2^k x 3 * 2^m) periodic grids: FP64 to
    1e-12 and FP32 to 2e-5 of the field maximum, as for 2^k sides."""
    rng = np.random.default_rng(nx * 11 + ny)
    sizes = (1.3, 0.7)
    s = cm.PeriodicFFTElasticHalfSpace((nx, ny), 1.1, sizes, precision=precision)
    f = rng.standard_normal((nx, ny))
    # FP64 at 6144: one transform buffer with the twiddles staged beside it
    assert _engine(s, precision) == 1
    o = oc.PeriodicSubstrate((nx, ny), 1.1, sizes)
    tol = 1e-12 if precision == "fp64" else 2e-5
    for op in ("evaluate_disp", "evaluate_force"):
        ref = getattr(o, op)(f)
        np.testing.assert_allclose(getattr(s, op)(f), ref, rtol=0, atol=tol * abs(ref).max(),
                                   err_msg=op)


@pytest.mark.parametrize("nx, ny", [(48, 48), (192, 96), (768, 768), (3072, 32)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_free_operator_vs_oracle(cm, nx, ny, precision):
    """Free grids (domains 96^2, 384 x 192, 1536^2, 6144 x 64) with padded
    and unpadded input, against the oracle with the extended-precision Love
    table (the tolerances of the power-of-two free grids)."""
    rng = np.random.default_rng(nx * 13 + ny)
    sizes = (1.3, 0.7)
    s = cm.FreeFFTElasticHalfSpace((nx, ny), 1.1, sizes, precision=precision)
    assert _engine(s, precision) == 1
    o = oc.FreeSubstrate((nx, ny), 1.1, sizes)
    ox = oc.FreeSubstrate((nx, ny), 1.1, sizes)
    ox.greens_function = oc.fft_forward(oc.love_kernel_extended((nx, ny), sizes, 1.1))
    for f in (rng.standard_normal((nx, ny)), rng.standard_normal((2 * nx, 2 * ny))):
        got = s.evaluate_disp(f)
        ref, exact = o.evaluate_disp(f), ox.evaluate_disp(f)
        assert got.shape == ref.shape
        if precision == "fp64":
            assert _rel(got, exact) < 1e-11, (f.shape, _rel(got, exact))
            assert _rel(got, ref) < _rel(ref, exact) + 1e-11, (f.shape, _rel(got, ref))
        else:
            assert _rel(got, exact) < 1e-6, (f.shape, _rel(got, exact))


CASES = [
    # kind, nb, hardness, external force
    ("periodic", (96, 96), None, 2e-3),
    ("periodic", (192, 384), None, 5e-3),
    ("periodic", (384, 384), 0.05, 5e-3),
    ("free", (96, 96), None, 2e-3),
    ("free", (48, 192), None, 1e-3),
    ("free", (3072, 32), None, 1e-4),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1][0]}x{c[1][1]}{'_plastic' if c[2] else ''}")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_vs_oracle(cm, case, precision):
    """FP64 within 1e-10 of the oracle's displacement with the same active
    set and offset; mixed within 1e-6 and the contact area within 1e-3."""
    kind, nb, hardness, F = case
    sizes = (1.0, 1.0)
    if kind == "free":
        h = oc.sphere(nb, sizes, 2.0)
        o = oc.FreeSubstrate(nb, 1.0, sizes)
        s = cm.FreeFFTElasticHalfSpace(nb, 1.0, sizes)
    else:
        h = oc.self_affine(nb, sizes, 0.7, 0.2 if hardness else 0.1, seed=23)
        o = oc.PeriodicSubstrate(nb, 1.0, sizes)
        s = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, sizes)
    assert _engine(s, "fp64") == 1 and _engine(s, "fp32") == 1
    kw = dict(external_force=F, pentol=1e-11 * (h.max() - h.min()), forcetol=1e-13, maxiter=5000)
    if hardness is not None:
        kw["hardness"] = hardness * o.area_per_pt
        kw["forcetol"] = 1e-10
    ref = oc.constrained_conjugate_gradients(o, h, **kw)
    res = cm.constrained_conjugate_gradients(s, h, precision=precision, **kw)
    assert res.success and ref["success"]
    x, xr = res.x[:nb[0], :nb[1]], ref["x"][:nb[0], :nb[1]]
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert _rel(x, xr) < tol, _rel(x, xr)
    if precision == "fp64":
        np.testing.assert_array_equal(res.active_set, ref["active_set"])
        np.testing.assert_allclose(res.offset, ref["offset"], rtol=1e-9)
    a, ar = np.count_nonzero(res.jac > 0), np.count_nonzero(ref["jac"] > 0)
    assert abs(a - ar) <= max(1, 1e-3 * ar)


def test_solve_twice_same_bits(cm):
    nb = (192, 96)
    h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=24)
    s = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    kw = dict(external_force=2e-3, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-10,
              precision="mixed")
    a = cm.constrained_conjugate_gradients(s, h, **kw)
    b = cm.constrained_conjugate_gradients(s, h, **kw)
    assert a.nit == b.nit
    for u, v in ((a.x, b.x), (a.jac, b.jac)):
        u = u.cpu().numpy() if hasattr(u, "cpu") else np.asarray(u)
        v = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
        assert np.array_equal(u.view(np.uint8), v.view(np.uint8))


def test_plastic_mixed_request_converges(cm):
    """A plastic request of the serving mix (periodic 1536^2, hardness 0.031
    E*, mean pressure 1.7e-4 E*) whose FP32 phase stops at its iteration cap:
    the mixed solve converges to the FP64 solution (within 1e-6), and its
    iteration count stays within maxiter."""
    from contactmechanics_b200.Generation import self_affine
    n = 1536
    h = torch.from_numpy(self_affine((n, n), (1.0, 1.0), 0.8, 0.1, seed=1000 * n)).cuda()
    p, hard = 0.00016841597410591723, 0.030904697985442438
    kw = dict(external_force=p, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-9 * p,
              maxiter=20000, hardness=hard / (n * n))
    s = cm.PeriodicFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
    ref = cm.constrained_conjugate_gradients(s, h, precision="fp64", **kw)
    res = cm.constrained_conjugate_gradients(s, h, precision="mixed", **kw)
    assert ref.success and res.success, res.message
    assert res.nit <= kw["maxiter"]
    x = res.x.cpu().numpy() if hasattr(res.x, "cpu") else np.asarray(res.x)
    xr = ref.x.cpu().numpy() if hasattr(ref.x, "cpu") else np.asarray(ref.x)
    assert _rel(x, xr) < 1e-6, _rel(x, xr)
