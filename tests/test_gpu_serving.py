"""Continuous batching: requests admitted while others run, admission by free
device memory, and each result the same alone and in the mix.

"Same" is bitwise between a request served alone and served among others
(same kernels, per-solve reductions); against the single-solve API the
mixed-precision results agree to 1e-6 relative displacement.
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


def _requests():
    reqs = []
    specs = [("periodic", (64, 96), 2e-3, None, None), ("periodic", (128, 64), 5e-3, None, None),
             ("free", (48, 40), None, 0.03, None), ("periodic", (64, 64), 4e-3, None, 0.05),
             ("periodic", (96, 96), 1e-3, None, None), ("free", (32, 48), 1e-3, None, None)]
    for i, (kind, nb, F, off, hard) in enumerate(specs):
        if kind == "free":
            h = oc.sphere(nb, (1.0, 1.0), 2.0)
        else:
            h = oc.self_affine(nb, (1.0, 1.0), 0.7, 0.2 if hard else 0.1, seed=60 + i)
        kw = dict(pentol=1e-11 * (h.max() - h.min()), forcetol=1e-13 if hard is None else 1e-10,
                  maxiter=5000)
        if F is not None:
            kw["external_force"] = F
        if off is not None:
            kw["offset"] = off
        if hard is not None:
            kw["hardness"] = hard * (1.0 / (nb[0] * nb[1]))
        reqs.append((kind, nb, h, kw))
    return reqs


def test_served_results_same_alone_and_in_the_mix(cm):
    from contactmechanics_b200.Serving import ContactServer
    reqs = _requests()
    srv = ContactServer(iters_per_step=4)
    try:
        first = [srv.submit(k, nb, (1.0, 1.0), h, **kw) for k, nb, h, kw in reqs[:3]]
        for _ in range(3):
            srv.step()  # the first requests are in flight ...
        later = [srv.submit(k, nb, (1.0, 1.0), h, **kw) for k, nb, h, kw in reqs[3:]]
        assert srv.n_active > 0 and srv.n_pending == len(later)
        srv.run_until_idle(timeout=120)  # ... when the later ones are admitted
        mixed = [r.result() for r in first + later]
    finally:
        srv.close()
    for (kind, nb, h, kw), rm in zip(reqs, mixed):
        assert rm.success
        alone_srv = ContactServer(iters_per_step=4)
        try:
            ra = alone_srv.submit(kind, nb, (1.0, 1.0), h, **kw)
            alone_srv.run_until_idle(timeout=120)
            ra = ra.result()
        finally:
            alone_srv.close()
        assert np.array_equal(ra.x, rm.x) and np.array_equal(ra.jac, rm.jac)
        assert ra.nit == rm.nit
        sub = (cm.FreeFFTElasticHalfSpace if kind == "free" else cm.PeriodicFFTElasticHalfSpace)(
            nb, 1.0, (1.0, 1.0))
        rs = cm.constrained_conjugate_gradients(sub, h, precision="fp64", **kw)
        xs = rs.x[:nb[0], :nb[1]]
        rel = np.linalg.norm(rm.x[:nb[0], :nb[1]] - xs) / np.linalg.norm(xs)
        assert rel < 1e-6, rel
        assert rm.latency_s is not None and rm.latency_s > 0


def test_admission_waits_for_free_device_memory(cm):
    from contactmechanics_b200.Serving import ContactServer
    free = {"bytes": 0}
    srv = ContactServer(mem_info=lambda: (free["bytes"], 1 << 40), hbm_reserve=1 << 20)
    try:
        kind, nb, h, kw = _requests()[0]
        r = srv.submit(kind, nb, (1.0, 1.0), h, **kw)
        srv.step()
        assert srv.n_active == 0 and srv.n_pending == 1   # no room: stays queued
        free["bytes"] = 1 << 40
        srv.run_until_idle(timeout=60)
        assert r.result().success
    finally:
        srv.close()


def test_cancel_pending_request(cm):
    from contactmechanics_b200.Serving import ContactServer
    srv = ContactServer(mem_info=lambda: (0, 1 << 40))
    try:
        kind, nb, h, kw = _requests()[1]
        r = srv.submit(kind, nb, (1.0, 1.0), h, **kw)
        assert srv.cancel(r)
        with pytest.raises(RuntimeError):
            r.result(timeout=1)
        assert srv.n_pending == 0
    finally:
        srv.close()


@pytest.mark.parametrize("threaded", [True, False])
def test_large_requests_take_the_single_solve_path(cm, threaded):
    """Requests of at least ``large_points`` domain points are solved one at a
    time by the single-solve path, concurrently with the batched small ones
    (or inline without the loop thread): their results equal
    constrained_conjugate_gradients bit for bit; the small ones stay within
    1e-6 of the FP64 single solve."""
    from contactmechanics_b200.Serving import ContactServer
    reqs = _requests()
    srv = ContactServer(iters_per_step=4, large_points=6000)
    try:
        if threaded:
            srv.start()
        handles = [srv.submit(k, nb, (1.0, 1.0), h, **kw) for k, nb, h, kw in reqs]
        if not threaded:
            srv.run_until_idle(timeout=120)
        results = [r.result(timeout=120) for r in handles]
    finally:
        srv.close()
    n_large = 0
    for (kind, nb, h, kw), rm in zip(reqs, results):
        assert rm.success and rm.latency_s > 0
        cls = cm.FreeFFTElasticHalfSpace if kind == "free" else cm.PeriodicFFTElasticHalfSpace
        sub = cls(nb, 1.0, (1.0, 1.0))
        points = (4 if kind == "free" else 1) * nb[0] * nb[1]
        if points >= 6000:
            n_large += 1
            rs = cm.constrained_conjugate_gradients(sub, h, precision="mixed", **kw)
            assert np.array_equal(rs.x, rm.x) and np.array_equal(rs.jac, rm.jac)
            assert rs.nit == rm.nit
        else:
            rs = cm.constrained_conjugate_gradients(sub, h, precision="fp64", **kw)
            xs = rs.x[:nb[0], :nb[1]]
            rel = np.linalg.norm(rm.x[:nb[0], :nb[1]] - xs) / np.linalg.norm(xs)
            assert rel < 1e-6, rel
    assert 0 < n_large < len(reqs)
