"""The oracle's SemiPeriodicFFTElasticHalfSpace restatement against the
reference's own outputs (tests/golden/semi_vectors.npz, written by
tests/golden/make_golden.py from the unmodified reference) and the
reference's known answers (test/test_fft_elastic_half_space.py:535-680)."""
import json
import os

import numpy as np
import pytest

from oracle import contact_oracle as oc

SEMI = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "semi_vectors.npz")
_npz = np.load(SEMI)
OPS = sorted(k[3:-7] for k in _npz.files if k.startswith("op_") and k.endswith("_config"))


def _sub(cfg, **kw):
    return oc.SemiPeriodicSubstrate(tuple(cfg["nb_grid_pts"]), cfg["young"],
                                    tuple(cfg["physical_sizes"]), tuple(cfg["periodicity"]),
                                    cfg["n_images"], **kw)


@pytest.mark.parametrize("name", OPS)
def test_semi_operator_vs_reference(name):
    cfg = json.loads(str(_npz[f"op_{name}_config"]))
    s = _sub(cfg)
    assert s.nb_domain_grid_pts == tuple(cfg["domain"])
    G = _npz[f"op_{name}_G"]
    np.testing.assert_allclose(s.greens_function, G, rtol=0, atol=1e-12 * abs(G).max())
    f, u = _npz[f"op_{name}_f"], _npz[f"op_{name}_u"]
    for key, got in (("disp", s.evaluate_disp(f)),
                     ("disp_full", s.evaluate_disp(f, bIncludePadding=True)),
                     ("force", s.evaluate_force(u)),
                     ("force_topo", s.evaluate_force(u[:f.shape[0], :f.shape[1]]))):
        ref = _npz[f"op_{name}_{key}"]
        assert got.shape == ref.shape, key
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-11 * abs(ref).max(), err_msg=key)


def test_semi_solve_vs_reference():
    cfg = json.loads(str(_npz["ccg_semi_ridge_config"]))
    s = _sub(cfg)
    h = _npz["ccg_semi_ridge_heights"]
    res = oc.constrained_conjugate_gradients(s, h, **cfg["solver_kwargs"])
    offset, fun, nit, nfev, success = _npz["ccg_semi_ridge_scalars"]
    assert res["success"] and success
    assert res["nit"] == int(nit)
    x = _npz["ccg_semi_ridge_x"]
    np.testing.assert_allclose(res["x"], x, rtol=0, atol=1e-10 * abs(x).max())
    np.testing.assert_array_equal(res["active_set"], _npz["ccg_semi_ridge_active_set"])


def test_semi_known_answers():
    """No images and no periodic axis: the free solution; swapping the
    periodic axis transposes the result (test_fft_elastic_half_space.py
    :585-605, 675-690)."""
    nb, sizes = (16, 16), (0.1, 0.1)
    f = np.zeros(nb)
    f[:8, :8] = 1e8
    semi = oc.SemiPeriodicSubstrate(nb, 210e9, sizes, (False, False), 0)
    free = oc.FreeSubstrate(nb, 210e9, sizes)
    ref = free.evaluate_disp(f)
    np.testing.assert_allclose(semi.evaluate_disp(f), ref, rtol=0, atol=1e-12 * abs(ref).max())
    for grid in [(32, 32), (32, 33), (33, 32)]:
        a = oc.SemiPeriodicSubstrate(grid, 210e9, sizes, (True, False), 10)
        b = oc.SemiPeriodicSubstrate(grid[::-1], 210e9, sizes, (False, True), 10)
        f = np.zeros(grid)
        f[:grid[0] // 2, :grid[1] // 2] = 1e8
        da, db = a.evaluate_disp(f), b.evaluate_disp(f.T).T
        np.testing.assert_allclose(da, db, rtol=0, atol=1e-12 * abs(da).max())
