"""k-space operators and energies, and the primal / dual objectives with
their Hessian products, on the device (FFTElasticHalfSpace.py:613-885,
Systems.py:459-1008).

* k-space operators, scalar product and energies against the reference's
  own outputs (tests/golden/kspace_vectors.npz) to 1e-12;
* the Hessian products are the exact change of the objectives' gradients
  (test/test_primal_dual_objective.py:166-213);
* L-BFGS-B on the primal and dual objectives reaches the Polonsky-Keer
  solution (test/test_primal_dual_objective.py:13-150, 215-254) within the
  reference's tolerances.
"""
import json
import os

import numpy as np
import pytest
import scipy.optimize as optim

from oracle import contact_oracle as oc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

KS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kspace_vectors.npz")
_npz = np.load(KS)
CASES = sorted(k[2:-7] for k in _npz.files if k.startswith("k_") and k.endswith("_config"))


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


@pytest.mark.parametrize("name", CASES)
def test_kspace_vs_reference(cm, name):
    cfg = json.loads(str(_npz[f"k_{name}_config"]))
    nb, sizes = tuple(cfg["nb_grid_pts"]), tuple(cfg["physical_sizes"])
    if cfg["kind"] == "free":
        s = cm.FreeFFTElasticHalfSpace(nb, cfg["young"], sizes)
    else:
        s = cm.PeriodicFFTElasticHalfSpace(nb, cfg["young"], sizes, **cfg["kwargs"])
    f, u = _npz[f"k_{name}_f"], _npz[f"k_{name}_u"]
    ka_ref, kb_ref = _npz[f"k_{name}_kdisp"], _npz[f"k_{name}_kforce"]
    for key, got in (("kdisp", s.evaluate_k_disp(f)), ("kforce", s.evaluate_k_force(u)),
                     ("kforce_k", s.evaluate_k_force_k(ka_ref))):
        ref = _npz[f"k_{name}_{key}"]
        assert got.shape == ref.shape, key
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * abs(ref).max(), err_msg=key)
    np.testing.assert_allclose(s.evaluate_scalar_product_k_space(ka_ref, kb_ref),
                               _npz[f"k_{name}_dot"], rtol=1e-12)
    np.testing.assert_allclose(s.evaluate(u, pot=True, forces=False)[0],
                               _npz[f"k_{name}_energy_k"], rtol=1e-12)
    e, fk = s.evaluate_k(ka_ref, pot=True, forces=True)
    np.testing.assert_allclose(e, _npz[f"k_{name}_evaluate_k_energy"], rtol=1e-12)
    # torch tensors in and out
    kt = s.evaluate_k_disp(torch.from_numpy(f).cuda())
    assert isinstance(kt, torch.Tensor) and kt.is_cuda
    np.testing.assert_allclose(kt.cpu().numpy(), ka_ref, rtol=0, atol=1e-12 * abs(ka_ref).max())


def _system(cm, nb, s, kind="periodic", R=10.0, Es=50.0):
    from contactmechanics_b200.Topography import Topography
    h = oc.sphere(nb, (s, s), R)
    cls = cm.PeriodicFFTElasticHalfSpace if kind == "periodic" else cm.FreeFFTElasticHalfSpace
    sub = cls(nb, Es, (s, s))
    return cm.NonSmoothContactSystem(sub, Topography(h, (s, s), periodic=kind == "periodic")), h


@pytest.mark.parametrize("s", [1.0, 2.0])
def test_primal_and_dual_hessians(cm, s):
    nx, ny = 64, 32
    system, _ = _system(cm, (nx, ny), s)
    rng = np.random.default_rng(5)
    gaps, dgaps = rng.random((nx, ny)), rng.random((nx, ny))
    obj = system.primal_objective(0, True)
    _, g0 = obj(gaps.reshape(-1))
    _, g1 = obj((gaps + dgaps).reshape(-1))
    np.testing.assert_allclose(system.primal_hessian_product(dgaps.reshape(-1)), g1 - g0,
                               rtol=1e-7, atol=1e-9 * abs(g1 - g0).max())
    obj = system.dual_objective(0, True)
    _, g0 = obj(gaps)
    _, g1 = obj(gaps + dgaps)
    np.testing.assert_allclose(system.dual_hessian_product(dgaps).reshape(g1.shape), g1 - g0,
                               rtol=1e-7, atol=1e-9 * abs(g1 - g0).max())


@pytest.mark.parametrize("s", [1.0, 2.0])
def test_primal_lbfgsb_vs_polonsky_keer(cm, s):
    n, offset = 64, 0.05
    system, h = _system(cm, (n, n), s)
    disp = h + offset
    res = system.primal_minimize_proxy(offset, init_gap=disp, solver="l-bfgs-b")
    assert res.success
    gap = res.x.reshape(n, n)
    pk = system.minimize_proxy(offset=offset, pentol=1e-10, forcetol=1e-12)
    assert pk.success
    gap_pk = pk.x - h - pk.offset
    np.testing.assert_allclose(gap, gap_pk, atol=1e-3)
    np.testing.assert_allclose(gap == 0, pk.jac > 0, atol=1e-3)


@pytest.mark.parametrize("s", [1.0, 2.0])
def test_dual_lbfgsb_vs_polonsky_keer(cm, s):
    n, offset = 64, 0.005
    system, h = _system(cm, (n, n), s)
    disp = np.maximum(h + offset, 0)
    init_force = system.substrate.evaluate_force(disp)
    res = system.dual_minimize_proxy(offset, init_force=init_force, solver="l-bfgs-b")
    assert res.success, res.message
    pk = system.minimize_proxy(offset=offset, pentol=1e-12, forcetol=1e-14)
    assert pk.success
    np.testing.assert_allclose(res.x.reshape(n, n), pk.jac, atol=1e-5)
    with pytest.raises(NotImplementedError):
        system.dual_minimize_proxy(offset, init_force=init_force, solver="ccg-with-restart")


@pytest.mark.parametrize("s", [1.0, 2.0])
def test_scipy_friendly_interface_nonperiodic(cm, s):
    """L-BFGS-B on ``objective`` with automatic bounds equals the
    Polonsky-Keer solution (test_primal_dual_objective.py:215-254)."""
    nx = ny = 32
    system, h = _system(cm, (nx, ny), s, kind="free")
    penetration = 0.005
    bnds = system._reshape_bounds(system._lbounds_from_heights(penetration))
    init_disp = np.ones(system.substrate.nb_subdomain_grid_pts)
    res = optim.minimize(system.objective(penetration, gradient=True),
                         system.shape_minimisation_input(init_disp), method="L-BFGS-B",
                         jac=True, bounds=bnds, options=dict(gtol=1e-8, ftol=1e-20))
    assert res.success
    lbfgsb = res.x.reshape((2 * nx, 2 * ny))
    pk = system.minimize_proxy(offset=penetration, pentol=1e-7)
    assert pk.success
    np.testing.assert_allclose(lbfgsb, pk.x, atol=1e-6)
