"""Parity of the CUDA path with the reference (golden vectors) and the oracle.

Tolerances: FP64 operators 1e-12 of the field's max; FP64 solves 1e-10
relative (the converged solution is unique for these convex problems);
FP32 operators 2e-5 relative to the field's max; mixed-precision solves
1e-6 relative in displacement and 1e-3 relative in contact area.
"""
import numpy as np
import pytest

from oracle import contact_oracle as oc
from tests.conftest import (GOLDEN, golden_config, golden_operator_config,
                            golden_operator_names, golden_solve_names)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

_npz = np.load(GOLDEN)


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def make_substrate(cm, cfg, precision="fp64"):
    nb, sizes = tuple(cfg["nb_grid_pts"]), tuple(cfg["physical_sizes"])
    if cfg["kind"] == "free":
        return cm.FreeFFTElasticHalfSpace(nb, cfg["young"], sizes, precision=precision)
    return cm.PeriodicFFTElasticHalfSpace(nb, cfg["young"], sizes, precision=precision,
                                          **cfg.get("kwargs", {}))


@pytest.mark.parametrize("name", golden_operator_names(_npz))
def test_operator_fp64_vs_reference(cm, golden, name):
    cfg = golden_operator_config(golden, name)
    s = make_substrate(cm, cfg)
    G = golden[f"op_{name}_G"]
    np.testing.assert_allclose(s.greens_function, G, rtol=0, atol=1e-13 * abs(G).max())
    ref = golden[f"op_{name}_disp"]
    out = s.evaluate_disp(golden[f"op_{name}_f"])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * abs(ref).max())
    ref = golden[f"op_{name}_force"]
    out = s.evaluate_force(golden[f"op_{name}_u"])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * abs(ref).max())
    if cfg["kind"] == "free":
        nx, ny = cfg["nb_grid_pts"]
        ref = golden[f"op_{name}_disp_unpadded"]
        out = s.evaluate_disp(golden[f"op_{name}_f"][:nx, :ny])
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * abs(ref).max())
        full = s.evaluate_disp(golden[f"op_{name}_f"][:nx, :ny], bIncludePadding=True)
        ref = golden[f"op_{name}_disp"]
        np.testing.assert_allclose(full, ref, rtol=0, atol=1e-12 * abs(ref).max())


@pytest.mark.parametrize("name", golden_operator_names(_npz))
def test_operator_fp32_vs_reference(cm, golden, name):
    cfg = golden_operator_config(golden, name)
    s = make_substrate(cm, cfg, precision="fp32")
    ref = golden[f"op_{name}_disp"]
    out = s.evaluate_disp(golden[f"op_{name}_f"])
    np.testing.assert_allclose(out, ref, rtol=0, atol=2e-5 * abs(ref).max())
    ref = golden[f"op_{name}_force"]
    out = s.evaluate_force(golden[f"op_{name}_u"])
    np.testing.assert_allclose(out, ref, rtol=0, atol=2e-5 * abs(ref).max())


@pytest.mark.parametrize("nx, ny", [(64, 64), (96, 192), (255, 256), (113, 65), (2048, 16),
                                     (8, 2048), (384, 350), (1, 7)])
def test_operator_sizes_vs_oracle(cm, nx, ny):
    """Mixed radices, prime factors (Bluestein-free direct stages), odd sizes."""
    rng = np.random.default_rng(nx * 1000 + ny)
    sizes = (1.3, 0.7)
    if nx == 1:
        s = cm.PeriodicFFTElasticHalfSpace((ny,), 1.1, (1.3,))
        o = oc.PeriodicSubstrate((ny,), 1.1, (1.3,))
        f = rng.standard_normal(ny)
    else:
        s = cm.PeriodicFFTElasticHalfSpace((nx, ny), 1.1, sizes)
        o = oc.PeriodicSubstrate((nx, ny), 1.1, sizes)
        f = rng.standard_normal((nx, ny))
    ref = o.evaluate_disp(f)
    np.testing.assert_allclose(s.evaluate_disp(f), ref, rtol=0, atol=1e-12 * abs(ref).max())
    ref = o.evaluate_force(f)
    np.testing.assert_allclose(s.evaluate_force(f), ref, rtol=0, atol=1e-12 * abs(ref).max())


@pytest.mark.parametrize("kind, nx, ny", [("periodic", 64, 64), ("periodic", 128, 512),
                                           ("periodic", 1024, 256), ("periodic", 2048, 2048),
                                           ("periodic", 4096, 64), ("free", 64, 128),
                                           ("free", 512, 512), ("free", 1024, 1024)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_operator_pow2_vs_oracle(cm, kind, nx, ny, precision):
    """Power-of-two domains (the by-value operator passes): square and
    rectangular periodic grids, free grids with padded and unpadded input
    (the unpadded input fills only a quarter of the domain's rows and
    columns).  Periodic: FP64 to 1e-12 and FP32 to 2e-5 of the field maximum.
    Free: the Love rectangle kernel sums corner terms that cancel, so the
    reference formula evaluated in FP64 is itself off by about r^2 eps at r
    pixels (||du|| / ||u|| of 3e-10 at 512^2, 2e-9 at 1024^2).  This library
    evaluates it in extended precision, so the FP64 result is checked against
    the oracle with an extended-precision table (||du||_2 / ||u||_2 < 1e-11;
    the extended evaluation itself keeps about 1e-12 of cancellation noise at
    a 2048^2 domain), and its distance to the plain FP64 oracle may not exceed
    that oracle's own error by more than 1e-11; FP32 to 1e-6."""
    rng = np.random.default_rng(nx * 7 + ny)
    sizes = (1.3, 0.7)
    tol = 1e-12 if precision == "fp64" else 2e-5
    if kind == "periodic":
        s = cm.PeriodicFFTElasticHalfSpace((nx, ny), 1.1, sizes, precision=precision)
        o = oc.PeriodicSubstrate((nx, ny), 1.1, sizes)
        f = rng.standard_normal((nx, ny))
        for op in ("evaluate_disp", "evaluate_force"):
            ref = getattr(o, op)(f)
            np.testing.assert_allclose(getattr(s, op)(f), ref, rtol=0, atol=tol * abs(ref).max(),
                                       err_msg=op)
    else:
        s = cm.FreeFFTElasticHalfSpace((nx, ny), 1.1, sizes, precision=precision)
        o = oc.FreeSubstrate((nx, ny), 1.1, sizes)
        ox = oc.FreeSubstrate((nx, ny), 1.1, sizes)
        ox.greens_function = oc.fft_forward(oc.love_kernel_extended((nx, ny), sizes, 1.1))
        for f in (rng.standard_normal((nx, ny)), rng.standard_normal((2 * nx, 2 * ny))):
            got = s.evaluate_disp(f)
            ref, exact = o.evaluate_disp(f), ox.evaluate_disp(f)
            assert got.shape == ref.shape

            def rel(u, v):
                return np.linalg.norm(u - v) / np.linalg.norm(v)
            if precision == "fp64":
                assert rel(got, exact) < 1e-11, (f.shape, rel(got, exact))
                assert rel(got, ref) < rel(ref, exact) + 1e-11, (f.shape, rel(got, ref))
            else:
                assert rel(got, exact) < 1e-6, (f.shape, rel(got, exact))


@pytest.mark.parametrize("nx, ny", [(8, 15), (8, 4), (9, 4), (113, 765)])
def test_sine_wave_force(cm, nx, ny):
    """Analytic p = -E*/2 |q| u (test/test_mpi_periodic_elastic_half_space.py:76-193)."""
    sx, sy, E = 2.45, 1.0, 1.0
    s = cm.PeriodicFFTElasticHalfSpace((nx, ny), E, (sx, sy))
    for k in [(1, 0), (0, 1), (1, 2), (nx // 2, 0), (1, ny // 2), (0, 2),
              (nx // 2, ny // 2), (0, ny // 2)]:
        qx, qy = k[0] * 2 * np.pi / sx, k[1] * 2 * np.pi / sy
        q = np.hypot(qx, qy)
        Y, X = np.meshgrid(np.linspace(0, sy, ny + 1)[:-1], np.linspace(0, sx, nx + 1)[:-1])
        disp = np.cos(qx * X + qy * Y) + np.sin(qx * X + qy * Y)
        p = s.evaluate_force(disp) / s.area_per_pt
        np.testing.assert_allclose(p, -disp * E / 2 * q, rtol=1e-7, atol=1e-10 * nx * ny)
        energy = s.evaluate(disp, pot=True, forces=False)[0]
        np.testing.assert_allclose(energy, E / 8 * 2 * q * sx * sy, rtol=1e-10)


def test_torch_zero_copy(cm):
    s = cm.PeriodicFFTElasticHalfSpace((64, 48), 1.0, (1.0, 1.0))
    f = torch.randn(64, 48, dtype=torch.float64, device="cuda")
    u = s.evaluate_disp(f)
    assert isinstance(u, torch.Tensor) and u.is_cuda
    ref = oc.PeriodicSubstrate((64, 48), 1.0, (1.0, 1.0)).evaluate_disp(f.cpu().numpy())
    np.testing.assert_allclose(u.cpu().numpy(), ref, rtol=0, atol=1e-12 * abs(ref).max())


def test_shape_error(cm):
    s = cm.PeriodicFFTElasticHalfSpace((16, 16), 1.0, (1.0, 1.0))
    with pytest.raises(cm.PeriodicFFTElasticHalfSpace.Error):
        s.evaluate_disp(np.zeros((16, 15)))
    free = cm.FreeFFTElasticHalfSpace((16, 16), 1.0, (1.0, 1.0))
    with pytest.raises(free.Error):
        free.evaluate_disp(np.zeros((16, 15)))


def _solve_golden(cm, golden, name, precision):
    cfg = golden_config(golden, name)
    h = golden[f"ccg_{name}_heights"]
    s = make_substrate(cm, cfg)
    kw = dict(cfg["solver_kwargs"])
    if cfg["hardness"] is not None:
        kw["hardness"] = cfg["hardness"] * s.area_per_pt
    return cfg, cm.constrained_conjugate_gradients(s, h, precision=precision, **kw)


@pytest.mark.parametrize("name", golden_solve_names(_npz))
def test_solve_fp64_vs_reference(cm, golden, name):
    cfg, res = _solve_golden(cm, golden, name, "fp64")
    offset, fun, nit, nfev, success = golden[f"ccg_{name}_scalars"]
    assert bool(res.success) == bool(success)
    x = golden[f"ccg_{name}_x"]
    jac = golden[f"ccg_{name}_jac"]
    if success:
        np.testing.assert_allclose(res.x, x, rtol=0, atol=1e-10 * abs(x).max())
        np.testing.assert_allclose(res.jac, jac, rtol=0, atol=1e-10 * abs(jac).max())
        np.testing.assert_array_equal(res.active_set, golden[f"ccg_{name}_active_set"])
        np.testing.assert_allclose(res.offset, offset, rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(res.fun, fun, rtol=1e-10)
        if f"ccg_{name}_plastic" in golden.files:
            np.testing.assert_array_equal(res.plastic, golden[f"ccg_{name}_plastic"])
    else:
        assert res.nit == int(nit)
        assert res.message == "Reached maxiter = {}".format(cfg["solver_kwargs"]["maxiter"])


@pytest.mark.parametrize("name", ["hertz_periodic_load", "sphere_free_load", "rough_periodic_load",
                                  "sphere_free_offset", "plastic_periodic_load"])
def test_solve_mixed_vs_reference(cm, golden, name):
    cfg, res = _solve_golden(cm, golden, name, "mixed")
    assert res.success
    x = golden[f"ccg_{name}_x"]
    nx, ny = cfg["nb_grid_pts"]
    rel = np.linalg.norm(res.x[:nx, :ny] - x[:nx, :ny]) / np.linalg.norm(x[:nx, :ny])
    assert rel <= 1e-6, rel
    a = np.count_nonzero(res.jac > 0)
    a_ref = np.count_nonzero(golden[f"ccg_{name}_jac"] > 0)
    assert abs(a - a_ref) <= 1e-3 * a_ref


P2_CASES = [
    # (kind, nb, hardness(pressure) or None, load F or None, offset or None)
    ("periodic", (64, 64), None, 2e-3, None),
    ("periodic", (128, 256), None, 5e-3, None),
    ("free", (64, 64), None, None, 0.02),
    ("free", (32, 64), None, 1e-3, None),
    ("periodic", (64, 64), 0.05, 4e-3, None),
]


def _oracle_case(kind, nb, hardness, F, offset, seed=21):
    sizes = (1.0, 1.0)
    if kind == "free":
        h = oc.sphere(nb, sizes, 2.0)
        o = oc.FreeSubstrate(nb, 1.0, sizes)
    else:
        h = oc.self_affine(nb, sizes, 0.7, 0.2 if hardness else 0.1, seed=seed)
        o = oc.PeriodicSubstrate(nb, 1.0, sizes)
    kw = dict(pentol=1e-11 * (h.max() - h.min()), forcetol=1e-13, maxiter=5000)
    if F is not None:
        kw["external_force"] = F
    if offset is not None:
        kw["offset"] = offset
    if hardness is not None:
        kw["hardness"] = hardness * o.area_per_pt
        kw["forcetol"] = 1e-10
    return h, o, kw


@pytest.mark.parametrize("case", P2_CASES, ids=lambda c: f"{c[0]}{c[1][0]}x{c[1][1]}{'_plastic' if c[2] else ''}")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_pow2_transforms_vs_oracle(cm, case, precision):
    """Sizes 64..256 run the register-resident power-of-two transforms."""
    kind, nb, hardness, F, offset = case
    h, o, kw = _oracle_case(*case)
    ref = oc.constrained_conjugate_gradients(o, h, **kw)
    if kind == "free":
        s = cm.FreeFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    else:
        s = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    res = cm.constrained_conjugate_gradients(s, h, precision=precision, **kw)
    assert res.success and ref["success"]
    x, xr = res.x[:nb[0], :nb[1]], ref["x"][:nb[0], :nb[1]]
    rel = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert rel < tol, rel
    if precision == "fp64":
        np.testing.assert_array_equal(res.active_set, ref["active_set"])
        np.testing.assert_allclose(res.offset, ref["offset"], rtol=1e-9)
    a, ar = np.count_nonzero(res.jac > 0), np.count_nonzero(ref["jac"] > 0)
    assert abs(a - ar) <= max(1, 1e-3 * ar)
