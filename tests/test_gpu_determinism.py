"""Every device path is deterministic: the same call twice gives the same
bits.  Reductions use fixed-order partials (no floating-point atomics), so
a rerun reproduces every sum, every step length and so every iterate; a
kernel that read uninitialised or racing memory would show up here as a
difference between runs.
"""
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


def _same(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("kind,nb", [("periodic", (128, 128)), ("periodic", (96, 80)),
                                     ("free", (64, 64)), ("free", (60, 45))])
def test_operator_twice(cm, kind, nb):
    cls = cm.PeriodicFFTElasticHalfSpace if kind == "periodic" else cm.FreeFFTElasticHalfSpace
    sub = cls(nb, 1.0, (1.0, 1.0))
    f = torch.from_numpy(np.random.default_rng(1).standard_normal(sub.nb_domain_grid_pts)).cuda()
    assert _same(sub.evaluate_disp(f), sub.evaluate_disp(f))
    assert _same(sub.evaluate_force(f), sub.evaluate_force(f))


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
@pytest.mark.parametrize("kind,nb,hard", [("periodic", (128, 128), None), ("free", (64, 64), None),
                                          ("periodic", (96, 96), 0.05)])
def test_solve_twice(cm, precision, kind, nb, hard):
    h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=21)
    cls = cm.PeriodicFFTElasticHalfSpace if kind == "periodic" else cm.FreeFFTElasticHalfSpace
    sub = cls(nb, 1.0, (1.0, 1.0))
    kw = dict(external_force=2e-3, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-10,
              maxiter=3000, precision=precision)
    if precision == "fp32":
        kw["pentol"] = 1e-5 * float(h.max() - h.min())
        kw["forcetol"] = 1e-7
    if hard is not None:
        kw["hardness"] = hard / (nb[0] * nb[1])
    a = cm.constrained_conjugate_gradients(sub, h, **kw)
    b = cm.constrained_conjugate_gradients(sub, h, **kw)
    assert a.nit == b.nit
    assert _same(a.x, b.x) and _same(a.jac, b.jac) and _same(a.active_set, b.active_set)
    assert a.offset == b.offset


@pytest.mark.parametrize("persistent", [0, 1])
def test_batch_twice(cm, persistent):
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    sizes = [(64, 96), (128, 64), (96, 96), (64, 64)]
    subs = [cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0)) for nb in sizes]
    hs = [oc.self_affine(nb, (1.0, 1.0), 0.7, 0.1, seed=30 + i) for i, nb in enumerate(sizes)]
    kw = dict(external_force=[2e-3] * 4, pentol=[1e-9 * float(h.max() - h.min()) for h in hs],
              forcetol=1e-10, precision="mixed")
    try:
        assert L.cm_tuning_set_batch_persistent(persistent) == 0
        a = cm.constrained_conjugate_gradients_batch(subs, hs, **kw)
        b = cm.constrained_conjugate_gradients_batch(subs, hs, **kw)
    finally:
        L.cm_tuning_set_batch_persistent(0)
    for ra, rb in zip(a, b):
        assert ra.nit == rb.nit
        assert _same(ra.x, rb.x) and _same(ra.jac, rb.jac)
