"""Parity at the benchmark's own configurations, against the oracle (GPU).

Each case solves one of the benchmark workloads (or a bounded sample of it)
on the device and compares with the FP64 oracle on the same seeded inputs:

* C1  rigid sphere R = 1 on a periodic 256^2 grid, L = 1, E* = 1, load
      1e-3 E* L^2 (FP64): against the oracle to 1e-10 and against Hertz
      (ReferenceSolutions/Hertz.py:104-131) within the reference's own
      tolerances (test/test_hertz.py:69-125: contact area to 10 %; here 3 %).
* C2  the first load of the benchmark sweep: free 1024^2 topography
      (2048^2 domain), self-affine H 0.8, slope 0.1, mean pressure 1e-4 E*.
      The oracle's Green's table is the Love kernel evaluated in extended
      precision (its FP64 evaluation carries about r^2 eps of cancellation
      error at r pixels, 2e-9 relative at this size; the library evaluates
      it in extended precision too).  FP64 to 1e-10; mixed precision to
      1e-6 in displacement and 1e-3 in contact area.
* C4  plastic periodic contact with the benchmark's surface parameters
      (H 0.7, slope 0.2, hardness 0.05 E*, mean pressure 5e-3 E*) on a
      512^2 grid (the 2048^2 benchmark size takes the oracle minutes on the
      host): displacement, plastic mask and the plastic displacement of
      PlasticNonSmoothContactSystem against the oracle.
* C3  eight solves of the batched benchmark's size mix (sides from
      {64, 96, 128, 192, 256, 384, 512}, the 96/192/384 sides on the
      mixed-radix transforms) through the batched solver (lockstep graph and
      persistent cluster kernel) and through the continuous-batching
      server, each against the oracle to 1e-6.

Tolerances are the benchmark's: pentol = 1e-9 (max h - min h), forcetol =
1e-12 F (C1: tighter, as in the reference's Hertz checks).
"""
import os

import numpy as np
import pytest

from oracle import contact_oracle as oc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

WORKERS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ---------------------------------------------------------------------------
# C1: Hertz, periodic 256^2, FP64
# ---------------------------------------------------------------------------
def test_c1_hertz_periodic_256(cm):
    n, L, R, F = 256, 1.0, 1.0, 1e-3
    h = oc.sphere((n, n), (L, L), R)
    kw = dict(external_force=F, pentol=1e-10 * float(h.max() - h.min()), forcetol=1e-14)
    sub = cm.PeriodicFFTElasticHalfSpace((n, n), 1.0, (L, L))
    res = cm.constrained_conjugate_gradients(sub, h, precision="fp64", **kw)
    ref = oc.constrained_conjugate_gradients(oc.PeriodicSubstrate((n, n), 1.0, (L, L), workers=WORKERS),
                                             h, **kw)
    assert res.success and ref["success"]
    assert rel(res.x, ref["x"]) < 1e-10
    np.testing.assert_array_equal(res.active_set, ref["active_set"])
    np.testing.assert_allclose(res.offset, ref["offset"], rtol=1e-10)
    # Hertz: a = R (3 F / (4 E* R^2))^(1/3), p0 = 3 F / (2 pi a^2)
    a = R * (3.0 / 4 * (F / (1.0 * R * R))) ** (1.0 / 3)
    p0 = 3 * F / (2 * np.pi * a * a)
    area_pt = (L / n) ** 2
    area = np.count_nonzero(res.jac > 0) * area_pt
    assert abs(area / (np.pi * a * a) - 1) < 0.03, area / (np.pi * a * a)
    pmax = float(res.jac.max()) / area_pt
    assert abs(pmax / p0 - 1) < 0.03, pmax / p0
    np.testing.assert_allclose(res.jac.sum(), F, rtol=1e-7)


# ---------------------------------------------------------------------------
# C2: first load of the free 1024^2 sweep
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2_case():
    from contactmechanics_b200.Generation import self_affine
    n = 1024
    h = self_affine((n, n), (1.0, 1.0), 0.8, 0.1, seed=2026, rolloff_wavelength=1.0 / 8)
    F = 1e-4
    kw = dict(external_force=F, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-12 * F)
    o = oc.FreeSubstrate((n, n), 1.0, (1.0, 1.0), workers=WORKERS)
    o.greens_function = oc.fft_forward(oc.love_kernel_extended((n, n), (1.0, 1.0), 1.0), WORKERS)
    o.surface_stiffness = oc.surface_stiffness(o.greens_function)
    ref = oc.constrained_conjugate_gradients(o, h, **kw)
    assert ref["success"]
    return n, h, kw, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c2_free_1024_first_load(cm, c2_case, precision):
    n, h, kw, ref = c2_case
    sub = cm.FreeFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
    res = cm.constrained_conjugate_gradients(sub, h, precision=precision, **kw)
    assert res.success
    e = rel(res.x[:n, :n], ref["x"][:n, :n])
    a, ar = np.count_nonzero(res.jac > 0), np.count_nonzero(ref["jac"] > 0)
    if precision == "fp64":
        assert e < 1e-10, e
        assert rel(res.x, ref["x"]) < 1e-10
        np.testing.assert_array_equal(res.active_set, ref["active_set"])
        assert abs(res.nit - ref["nit"]) <= 2, (res.nit, ref["nit"])
    else:
        assert e < 1e-6, e
        assert abs(a - ar) <= 1e-3 * ar, (a, ar)
    np.testing.assert_allclose(res.jac.sum(), kw["external_force"], rtol=1e-6)


# ---------------------------------------------------------------------------
# C4: plastic periodic contact (benchmark surface parameters, 512^2)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c4_case():
    from contactmechanics_b200.Generation import self_affine
    n = 512
    h = self_affine((n, n), (1.0, 1.0), 0.7, 0.2, seed=4)
    F, H = 5e-3, 0.05
    kw = dict(external_force=F, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-9 * F,
              maxiter=20000)
    o = oc.PeriodicSubstrate((n, n), 1.0, (1.0, 1.0), workers=WORKERS)
    ref = oc.constrained_conjugate_gradients(o, h, hardness=H * o.area_per_pt, **kw)
    assert ref["success"]
    # the plastic system adds the (negative) gap of the plastic points to the
    # plastic displacement (PlasticSystemSpecialisations.py:60-69)
    gap = ref["x"][:n, :n] - (h + ref["offset"])
    ref["plastic_displ"] = np.where(ref["plastic"], gap, 0.0)
    return n, h, F, H, kw, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c4_plastic_periodic(cm, c4_case, precision):
    n, h, F, H, kw, ref = c4_case
    from contactmechanics_b200.Topography import PlasticTopography, Topography
    topo = PlasticTopography(Topography(h, (1.0, 1.0)), H)
    system = cm.make_plastic_system(topo, substrate="periodic", young=1.0)
    res = system.minimize_proxy(precision=precision, **kw)
    assert res.success
    e = rel(res.x, ref["x"])
    npl, npl_ref = int(np.count_nonzero(res.plastic)), int(np.count_nonzero(ref["plastic"]))
    assert npl_ref > 0
    pd, pd_ref = topo.plastic_displ, ref["plastic_displ"]
    if precision == "fp64":
        assert e < 1e-10, e
        np.testing.assert_array_equal(res.plastic, ref["plastic"])
        np.testing.assert_array_equal(res.active_set, ref["active_set"])
        assert rel(pd, pd_ref) < 1e-9
    else:
        assert e < 1e-6, e
        a, ar = np.count_nonzero(res.jac > 0), np.count_nonzero(ref["jac"] > 0)
        assert abs(a - ar) <= 1e-3 * ar
        assert rel(pd, pd_ref) < 1e-5
        # The plastic flag is the sign of a gap; at the rim of the flowing
        # region gaps sit at the convergence tolerance, so a solve that
        # reaches the same tolerances along another path (FP32, then FP64)
        # may flag a few rim points differently.  Every mismatch lies on the
        # rim (a point whose 4-neighbourhood holds both flags), and they are
        # a small fraction of the plastic area.
        pl, pl_ref = np.asarray(res.plastic, bool), np.asarray(ref["plastic"], bool)
        rim = np.zeros_like(pl_ref)
        for m in (pl_ref, pl):
            for ax in (0, 1):
                for sh in (1, -1):
                    rim |= m != np.roll(m, sh, axis=ax)
        mism = pl != pl_ref
        assert not np.any(mism & ~rim), int(np.count_nonzero(mism & ~rim))
        assert abs(npl - npl_ref) <= 5e-3 * npl_ref, (npl, npl_ref)
    assert float(res.jac.max()) <= H * (1.0 / n) ** 2 * (1 + 1e-12)


# ---------------------------------------------------------------------------
# C3 size mix: batched solver and continuous-batching server
# ---------------------------------------------------------------------------
C3_SHAPES = [(96, 384), (192, 64), (384, 192), (512, 96), (64, 512), (256, 384), (128, 192),
             (384, 384)]


@pytest.fixture(scope="module")
def c3_cases():
    from contactmechanics_b200.Generation import self_affine
    cases = []
    for i, nb in enumerate(C3_SHAPES):
        rng = np.random.default_rng(100 + i)
        hurst, slope = rng.uniform(0.3, 0.9), rng.uniform(0.05, 0.2)
        F = float(10 ** rng.uniform(-4, -2))
        h = self_affine(nb, (1.0, 1.0), hurst, slope, seed=100 + i)
        kw = dict(external_force=F, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-12 * F)
        ref = oc.constrained_conjugate_gradients(
            oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0), workers=WORKERS), h, **kw)
        assert ref["success"]
        cases.append((nb, h, kw, ref))
    return cases


@pytest.mark.parametrize("persistent", [0, 1], ids=["lockstep", "persistent"])
def test_c3_size_mix_batched_vs_oracle(cm, c3_cases, persistent):
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    subs = [cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0)) for nb, _, _, _ in c3_cases]
    try:
        assert L.cm_tuning_set_batch_persistent(persistent) == 0
        res = cm.constrained_conjugate_gradients_batch(
            subs, [h for _, h, _, _ in c3_cases],
            external_force=[kw["external_force"] for _, _, kw, _ in c3_cases],
            pentol=[kw["pentol"] for _, _, kw, _ in c3_cases],
            forcetol=[kw["forcetol"] for _, _, kw, _ in c3_cases], precision="mixed")
    finally:
        L.cm_tuning_set_batch_persistent(0)
    for (nb, h, kw, ref), r in zip(c3_cases, res):
        assert r.success
        e = rel(r.x, ref["x"])
        assert e < 1e-6, (nb, e)
        a, ar = np.count_nonzero(r.jac > 0), np.count_nonzero(ref["jac"] > 0)
        assert abs(a - ar) <= max(1, 1e-3 * ar), (nb, a, ar)


def test_c3_size_mix_served_vs_oracle(cm, c3_cases):
    from contactmechanics_b200.Serving import ContactServer
    srv = ContactServer(iters_per_step=8)
    try:
        handles = [srv.submit("periodic", nb, (1.0, 1.0), h, **kw) for nb, h, kw, _ in c3_cases]
        srv.run_until_idle(timeout=300)
        out = [hd.result() for hd in handles]
    finally:
        srv.close()
    for (nb, h, kw, ref), r in zip(c3_cases, out):
        assert r.success
        e = rel(np.asarray(r.x), ref["x"])
        assert e < 1e-6, (nb, e)
