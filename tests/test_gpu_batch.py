"""Batched solves: each member of a batch equals its solve alone.

Both batch paths are covered: the persistent cluster kernel (elastic
batches, one launch for the whole batch) and the lockstep per-pass kernels
(any batch; plastic batches always take it).  FP64 batch members agree with
the single-solve path to 1e-10 (relative displacement) with identical
active sets; a member's result is bitwise the same whether it is solved in
a batch of one or among other solves; mixed precision members are within
1e-6 of the FP64 oracle.
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


CASES = [
    # kind, nb, hurst, slope, F (load) or None, offset, hardness (pressure)
    ("periodic", (64, 96), 0.8, 0.1, 2e-3, None, None),
    ("periodic", (96, 64), 0.5, 0.15, 4e-3, None, None),
    ("periodic", (128, 128), 0.7, 0.1, 1e-3, None, None),
    ("free", (48, 40), None, None, None, 0.03, None),
    ("periodic", (64, 64), 0.7, 0.2, 4e-3, None, 0.05),
]


ELASTIC = [c for c in CASES if c[6] is None]


@pytest.fixture(params=["persistent", "lockstep"])
def path(request, cm):
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    assert L.cm_tuning_set_batch_persistent(1 if request.param == "persistent" else 0) == 0
    yield request.param
    L.cm_tuning_set_batch_persistent(0)


def _cases(path):
    # a plastic member sends a batch to the lockstep kernels
    return ELASTIC if path == "persistent" else CASES


def _problem(cm, case, seed):
    kind, nb, hurst, slope, F, off, hard = case
    sizes = (1.0, 1.0)
    if kind == "free":
        h = oc.sphere(nb, sizes, 2.0)
        sub = cm.FreeFFTElasticHalfSpace(nb, 1.0, sizes)
        o = oc.FreeSubstrate(nb, 1.0, sizes)
    else:
        h = oc.self_affine(nb, sizes, hurst, slope, seed=seed)
        sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, sizes)
        o = oc.PeriodicSubstrate(nb, 1.0, sizes)
    kw = dict(pentol=1e-11 * (h.max() - h.min()), forcetol=1e-13 if hard is None else 1e-10,
              maxiter=5000)
    if F is not None:
        kw["external_force"] = F
    if off is not None:
        kw["offset"] = off
    if hard is not None:
        kw["hardness"] = hard * o.area_per_pt
    return sub, o, h, kw


def _batch(cm, problems, precision):
    subs = [p[0] for p in problems]
    hs = [p[2] for p in problems]
    keys = ["external_force", "offset", "hardness", "pentol", "forcetol"]
    kw = {k: [p[3].get(k) for p in problems] for k in keys}
    if all(v is None for v in kw["hardness"]):
        kw["hardness"] = None
    return cm.constrained_conjugate_gradients_batch(subs, hs, precision=precision, maxiter=5000, **kw)


def test_batch_fp64_matches_single_solves(cm, path):
    problems = [_problem(cm, c, seed=30 + i) for i, c in enumerate(_cases(path))]
    batch = _batch(cm, problems, "fp64")
    for (sub, o, h, kw), rb in zip(problems, batch):
        rs = cm.constrained_conjugate_gradients(sub, h, precision="fp64", **kw)
        assert rb.success and rs.success
        nb = sub.nb_grid_pts
        rel = np.linalg.norm(rb.x[:nb[0], :nb[1]] - rs.x[:nb[0], :nb[1]]) / \
            np.linalg.norm(rs.x[:nb[0], :nb[1]])
        assert rel < 1e-10, rel
        np.testing.assert_array_equal(rb.active_set, rs.active_set)


def test_batch_member_same_alone_and_in_the_mix(cm, path):
    cases = _cases(path)
    problems = [_problem(cm, c, seed=40 + i) for i, c in enumerate(cases)]
    mixed = _batch(cm, problems, "mixed")
    ks = (0, 3, 4) if path == "lockstep" else range(len(cases))
    for k in ks:
        alone = _batch(cm, [problems[k]], "mixed")[0]
        assert np.array_equal(alone.x, mixed[k].x)
        assert np.array_equal(alone.jac, mixed[k].jac)
        assert alone.nit == mixed[k].nit


def test_batch_mixed_vs_oracle(cm, path):
    problems = [_problem(cm, c, seed=50 + i) for i, c in enumerate(_cases(path))]
    batch = _batch(cm, problems, "mixed")
    for (sub, o, h, kw), rb in zip(problems, batch):
        ref = oc.constrained_conjugate_gradients(o, h, **kw)
        assert rb.success and ref["success"]
        nb = sub.nb_grid_pts
        xr = ref["x"][:nb[0], :nb[1]]
        rel = np.linalg.norm(rb.x[:nb[0], :nb[1]] - xr) / np.linalg.norm(xr)
        assert rel < 1e-6, rel
        a, ar = np.count_nonzero(rb.jac > 0), np.count_nonzero(ref["jac"] > 0)
        assert abs(a - ar) <= max(1, 1e-3 * ar)


def test_batch_under_other_launch_shapes(cm):
    """Batched results do not depend on the tuned tile sizes and block
    threads beyond rounding: extreme choices still match the oracle."""
    from contactmechanics_b200 import Autotune
    try:
        Autotune.apply({"tiles": {"fp64": {"64": 512, "96": 512, "128": 512}},
                        "threads": {"fp64": 128}})
        probs = [_problem(cm, c, 40 + i) for i, c in enumerate(CASES[:3])]  # plans under the shapes
        res = _batch(cm, probs, "fp64")
    finally:
        Autotune.clear()
        Autotune._applied = False
        Autotune.apply_default()
    for (sub, o, h, kw), r in zip(probs, res):
        ref = oc.constrained_conjugate_gradients(o, h, **kw)
        assert r.success and ref["success"]
        np.testing.assert_allclose(r.x, ref["x"], rtol=0, atol=1e-10 * abs(ref["x"]).max())


def test_persistent_batch_is_one_launch(cm):
    """An elastic batch (FP32 phase, FP64 refinement and results of every
    solve) is one kernel launch of the library."""
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    problems = [_problem(cm, c, seed=60 + i) for i, c in enumerate(ELASTIC)]
    try:
        assert L.cm_tuning_set_batch_persistent(1) == 0
        _batch(cm, problems, "mixed")  # plans' solver buffers allocated
        before = L.cm_launch_count()
        res = _batch(cm, problems, "mixed")
        assert L.cm_launch_count() - before == 1
    finally:
        L.cm_tuning_set_batch_persistent(0)
    assert all(r.success for r in res)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
def test_persistent_and_lockstep_agree(cm, precision):
    """The two batch paths reach the same solutions (to the precision's
    rounding) with the same iteration counts up to a couple of steps."""
    from contactmechanics_b200 import _lib
    L = _lib.lib()
    problems = [_problem(cm, c, seed=70 + i) for i, c in enumerate(ELASTIC)]
    if precision == "fp32":
        # tolerances an FP32 solve reaches; offset control's test on the
        # relative change of the total force (thermotol) is below FP32
        # rounding, so only the load-controlled solves
        problems = [p for p, c in zip(problems, ELASTIC) if c[4] is not None]
        for sub, o, h, kw in problems:
            kw["pentol"] = 1e-5 * float(h.max() - h.min())
            kw["forcetol"] = 1e-7
    lock = _batch(cm, problems, precision)
    try:
        assert L.cm_tuning_set_batch_persistent(1) == 0
        pers = _batch(cm, problems, precision)
    finally:
        L.cm_tuning_set_batch_persistent(0)
    tol = {"fp64": 1e-10, "mixed": 1e-6, "fp32": 1e-4}[precision]
    for (sub, o, h, kw), a, b in zip(problems, pers, lock):
        assert a.success and b.success
        nb = sub.nb_grid_pts
        xa, xb = a.x[:nb[0], :nb[1]], b.x[:nb[0], :nb[1]]
        assert np.linalg.norm(xa - xb) / np.linalg.norm(xb) < tol
        assert abs(a.nit - b.nit) <= 3, (a.nit, b.nit)

