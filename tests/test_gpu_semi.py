"""SemiPeriodicFFTElasticHalfSpace on the device against the reference's own
outputs (tests/golden/semi_vectors.npz) and the oracle.

The library sums the periodic images of the Love kernel in extended
precision; the reference sums them in FP64, where the far images cancel by
about r^2 eps (r the image distance in pixels, up to 10 periods), so the
reference's own table carries errors of about 1e-11 of its maximum at these
sizes (1.3e-10 at 33 x 32): tables and operators agree with the oracle's
extended-precision sum to 1e-12 of the field maximum and are no farther from
the reference than the reference's own FP64 error plus 1e-11; the solve
agrees with the reference to 1e-9.
"""
import json
import os

import numpy as np
import pytest

from oracle import contact_oracle as oc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SEMI = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "semi_vectors.npz")
_npz = np.load(SEMI)
OPS = sorted(k[3:-7] for k in _npz.files if k.startswith("op_") and k.endswith("_config"))


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def _make(cm, cfg, **kw):
    return cm.SemiPeriodicFFTElasticHalfSpace(tuple(cfg["nb_grid_pts"]), cfg["young"],
                                              tuple(cfg["physical_sizes"]),
                                              periodicity=tuple(cfg["periodicity"]),
                                              n_images=cfg["n_images"], **kw)


@pytest.mark.parametrize("name", OPS)
def test_semi_operator_vs_reference(cm, name):
    cfg = json.loads(str(_npz[f"op_{name}_config"]))
    s = _make(cm, cfg)
    assert s.nb_domain_grid_pts == tuple(cfg["domain"])
    args = (tuple(cfg["nb_grid_pts"]), cfg["young"], tuple(cfg["physical_sizes"]),
            tuple(cfg["periodicity"]), cfg["n_images"])
    o64 = oc.SemiPeriodicSubstrate(*args)                 # the reference's FP64 image sum
    oxt = oc.SemiPeriodicSubstrate(*args, extended=True)  # the image sum evaluated exactly
    G = _npz[f"op_{name}_G"]
    np.testing.assert_allclose(s.greens_function, oxt.greens_function, rtol=0,
                               atol=1e-12 * abs(G).max())
    f, u = _npz[f"op_{name}_f"], _npz[f"op_{name}_u"]
    ut = u[:f.shape[0], :f.shape[1]]
    for key, fn, arg in (("disp", lambda o, a: o.evaluate_disp(a), f),
                         ("disp_full", lambda o, a: o.evaluate_disp(a, bIncludePadding=True), f),
                         ("force", lambda o, a: o.evaluate_force(a), u),
                         ("force_topo", lambda o, a: o.evaluate_force(a), ut)):
        ref = _npz[f"op_{name}_{key}"]
        got = fn(s, arg)
        assert got.shape == ref.shape, key
        exact = fn(oxt, arg)
        scale = abs(ref).max()
        # exact to rounding; and no farther from the reference than the
        # reference's own FP64 image-sum error
        assert abs(got - exact).max() <= 1e-12 * scale, key
        own = abs(fn(o64, arg) - exact).max()
        assert abs(got - ref).max() <= own + 1e-11 * scale, key
    np.testing.assert_allclose(s.G_real, oxt.G_real, rtol=0, atol=1e-12 * abs(oxt.G_real).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_semi_solve_vs_reference(cm, precision):
    cfg = json.loads(str(_npz["ccg_semi_ridge_config"]))
    s = _make(cm, cfg)
    h = _npz["ccg_semi_ridge_heights"]
    res = cm.constrained_conjugate_gradients(s, h, precision=precision, **cfg["solver_kwargs"])
    assert res.success
    x = _npz["ccg_semi_ridge_x"]
    rel = np.linalg.norm(res.x - x) / np.linalg.norm(x)
    assert rel < (1e-9 if precision == "fp64" else 1e-6), rel
    if precision == "fp64":
        np.testing.assert_array_equal(res.active_set, _npz["ccg_semi_ridge_active_set"])
        offset, fun, nit, nfev, success = _npz["ccg_semi_ridge_scalars"]
        np.testing.assert_allclose(res.offset, offset, rtol=1e-9)


def test_semi_known_answers(cm):
    """No images and no periodic axis: the free solution; swapping the
    periodic axis transposes the result (test_fft_elastic_half_space.py
    :585-605, 675-690)."""
    nb, sizes = (16, 16), (0.1, 0.1)
    f = np.zeros(nb)
    f[:8, :8] = 1e8
    semi = cm.SemiPeriodicFFTElasticHalfSpace(nb, 210e9, sizes, periodicity=(False, False),
                                              n_images=0)
    ref = cm.FreeFFTElasticHalfSpace(nb, 210e9, sizes).evaluate_disp(f)
    np.testing.assert_allclose(semi.evaluate_disp(f), ref, rtol=0, atol=1e-12 * abs(ref).max())
    for grid in [(32, 32), (32, 33), (33, 32)]:
        a = cm.SemiPeriodicFFTElasticHalfSpace(grid, 210e9, sizes, periodicity=(True, False))
        b = cm.SemiPeriodicFFTElasticHalfSpace(grid[::-1], 210e9, sizes, periodicity=(False, True))
        f = np.zeros(grid)
        f[:grid[0] // 2, :grid[1] // 2] = 1e8
        da, db = a.evaluate_disp(f), b.evaluate_disp(f.T).T
        np.testing.assert_allclose(da, db, rtol=0, atol=1e-12 * abs(da).max())
