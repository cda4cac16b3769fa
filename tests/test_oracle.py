"""Pin the CPU oracle against the reference.

The golden vectors in ``tests/golden/reference_vectors.npz`` were produced by
running the reference's own code (``tests/golden/make_golden.py``).  The
analytic cases re-derive the reference's known-answer tests
(test/test_mpi_periodic_elastic_half_space.py:76-193, test/ReferenceSolutions/
test_reference_solutions.py:84-93, test/test_hertz.py:39-205).
"""
import numpy as np
import pytest

from oracle import contact_oracle as oc
from tests.conftest import (GOLDEN, PIPELINE_OUTPUTS, golden_config, golden_operator_config,
                            golden_operator_names, golden_pipeline_case, golden_pipeline_names,
                            golden_solve_names)

_npz = np.load(GOLDEN)


def make_oracle_substrate(cfg):
    nb, sizes = tuple(cfg["nb_grid_pts"]), tuple(cfg["physical_sizes"])
    if cfg["kind"] == "free":
        return oc.FreeSubstrate(nb, cfg["young"], sizes)
    return oc.PeriodicSubstrate(nb, cfg["young"], sizes, **cfg.get("kwargs", {}))


@pytest.mark.parametrize("name", golden_operator_names(_npz))
def test_operator_matches_reference(golden, name):
    cfg = golden_operator_config(golden, name)
    s = make_oracle_substrate(cfg)
    G = golden[f"op_{name}_G"]
    np.testing.assert_allclose(s.greens_function, G, rtol=1e-13,
                               atol=1e-13 * abs(G).max())
    disp = s.evaluate_disp(golden[f"op_{name}_f"])
    ref = golden[f"op_{name}_disp"]
    np.testing.assert_allclose(disp, ref, rtol=0, atol=1e-12 * abs(ref).max())
    force = s.evaluate_force(golden[f"op_{name}_u"])
    ref = golden[f"op_{name}_force"]
    np.testing.assert_allclose(force, ref, rtol=0, atol=1e-12 * abs(ref).max())
    if cfg["kind"] == "free":
        nx, ny = cfg["nb_grid_pts"]
        un = s.evaluate_disp(golden[f"op_{name}_f"][:nx, :ny])
        ref = golden[f"op_{name}_disp_unpadded"]
        np.testing.assert_allclose(un, ref, rtol=0, atol=1e-12 * abs(ref).max())


def run_oracle_solve(cfg, heights):
    s = make_oracle_substrate(cfg)
    kw = dict(cfg["solver_kwargs"])
    hardness = cfg["hardness"]
    if hardness is not None:
        kw["hardness"] = hardness * s.area_per_pt
    return s, oc.constrained_conjugate_gradients(s, heights, **kw)


@pytest.mark.parametrize("name", golden_solve_names(_npz))
def test_solve_matches_reference(golden, name):
    cfg = golden_config(golden, name)
    h = golden[f"ccg_{name}_heights"]
    s, res = run_oracle_solve(cfg, h)
    offset, fun, nit, nfev, success = golden[f"ccg_{name}_scalars"]
    assert bool(res["success"]) == bool(success)
    assert res["nit"] == int(nit)
    assert res["nfev"] == int(nfev)
    x = golden[f"ccg_{name}_x"]
    np.testing.assert_allclose(res["x"], x, rtol=0, atol=1e-11 * abs(x).max())
    jac = golden[f"ccg_{name}_jac"]
    np.testing.assert_allclose(res["jac"], jac, rtol=0, atol=1e-11 * abs(jac).max())
    np.testing.assert_array_equal(res["active_set"], golden[f"ccg_{name}_active_set"])
    np.testing.assert_allclose(res["offset"], offset, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(res["fun"], fun, rtol=1e-10)
    if f"ccg_{name}_plastic" in golden.files:
        np.testing.assert_array_equal(res["plastic"], golden[f"ccg_{name}_plastic"])
    if not success:
        assert res["message"] == "Reached maxiter = {}".format(cfg["solver_kwargs"]["maxiter"])


@pytest.mark.parametrize("nx, ny", [(8, 15), (8, 4), (9, 4), (113, 65)])
def test_sine_wave_force_analytic(nx, ny):
    """p = -E*/2 |q| u for a sinusoidal displacement, including the Nyquist
    edges (test/test_mpi_periodic_elastic_half_space.py:76-193)."""
    sx, sy, E = 2.45, 1.0, 1.0
    s = oc.PeriodicSubstrate((nx, ny), E, (sx, sy))
    for k in [(1, 0), (0, 1), (1, 2), (nx // 2, 0), (1, ny // 2), (0, 2),
              (nx // 2, ny // 2), (0, ny // 2)]:
        qx, qy = k[0] * 2 * np.pi / sx, k[1] * 2 * np.pi / sy
        q = np.hypot(qx, qy)
        Y, X = np.meshgrid(np.linspace(0, sy, ny + 1)[:-1], np.linspace(0, sx, nx + 1)[:-1])
        disp = np.cos(qx * X + qy * Y) + np.sin(qx * X + qy * Y)
        p = s.evaluate_force(disp) / s.area_per_pt
        np.testing.assert_allclose(p, -disp * E / 2 * q, rtol=1e-7, atol=1e-10 * nx * ny)
        energy = 0.5 * np.sum(-s.evaluate_force(disp) * disp)
        np.testing.assert_allclose(energy, E / 8 * 2 * q * sx * sy, rtol=1e-10)


@pytest.mark.parametrize("res", [(32, 32), (33, 32), (32, 33), (64,)])
def test_force_disp_reversibility(res):
    """Zero-mean fields survive force->disp->force (test/test_fft_elastic_half_space.py:132-158)."""
    rng = np.random.default_rng(3)
    s = oc.PeriodicSubstrate(res, 1.3, (1.0, 2.0)[:len(res)])
    d = rng.random(res)
    d -= d.mean()
    assert np.mean(abs(d - s.evaluate_disp(s.evaluate_force(d)))) < 1e-10
    f = rng.random(res)
    f -= f.mean()
    assert np.mean(abs(f - s.evaluate_force(s.evaluate_disp(f)))) < 1e-10


def test_hertz_known_answer():
    """test/ReferenceSolutions/test_reference_solutions.py:84-93."""
    Es, R, F = 5.0, 4.0, 7.0
    d = (9 * F ** 2 / (16 * R * Es ** 2)) ** (1 / 3)
    np.testing.assert_allclose(d, 0.6507879989531481, rtol=1e-7)
    a = R * (3.0 / 4 * (F / (Es * R ** 2))) ** (1.0 / 3)
    p0 = 3 * F / (2 * np.pi * a * a)
    np.testing.assert_allclose((a, p0), (1.6134286460245437, 1.2839257217043503), rtol=1e-7)


def test_free_hertz_against_theory():
    """Free sphere under load: offset and contact area against Hertz
    (test/test_hertz.py:39-125, smaller grid)."""
    nx = ny = 64
    sx, R, E, F = 5.0, 20.0, 102.0, 15.0
    s = oc.FreeSubstrate((nx, ny), E, (sx, sx))
    h = oc.sphere((nx, ny), (sx, sx), R)
    res = oc.constrained_conjugate_gradients(s, h, external_force=F)
    assert res["success"]
    np.testing.assert_allclose(res["jac"].sum(), F, rtol=1e-7)
    d = (9 * F ** 2 / (16 * R * E ** 2)) ** (1 / 3)
    np.testing.assert_allclose(res["offset"], d, rtol=5e-2)
    a = R * (3.0 / 4 * (F / (E * R ** 2))) ** (1.0 / 3)
    area = np.count_nonzero(res["jac"] > 0) * s.area_per_pt
    np.testing.assert_allclose(area, np.pi * a * a, rtol=0.2)


def test_free_boundary_check():
    s = oc.FreeSubstrate((8, 8), 1.0, (1.0, 1.0))
    f = np.zeros((8, 8))
    s.check_boundaries(f)
    f[0, 3] = 1.0
    with pytest.raises(oc.FreeBoundaryError):
        s.check_boundaries(f)


def test_shape_error():
    s = oc.PeriodicSubstrate((8, 8), 1.0, (1.0, 1.0))
    with pytest.raises(oc.SubstrateError):
        s.evaluate_disp(np.zeros((8, 9)))


def test_love_kernel_extended_precision():
    """The extended-precision evaluation of the Love kernel agrees with the
    FP64 one to the cancellation error of the FP64 formula (about r^2 eps at
    r pixels from the load): tight on a small grid, looser on a larger one."""
    for n, tol in ((8, 1e-13), (64, 1e-11)):
        a = oc.love_kernel((n, n), (1.3, 0.7), 1.1)
        b = oc.love_kernel_extended((n, n), (1.3, 0.7), 1.1)
        assert a.shape == b.shape
        assert abs(a - b).max() <= tol * abs(b).max()


@pytest.mark.parametrize("name", golden_pipeline_names(_npz))
def test_pipeline_oracle_vs_reference(golden, name):
    """The restated automated sweep reproduces the reference's
    contact_mechanics: per-step means, areas and convergence flags, and the
    last step's fields."""
    h, sizes, periodic, kw = golden_pipeline_case(golden, name)
    opt = kw.pop("optimizer_kwargs", {})
    last = {}

    def cb(disp, gap, pressure, contacting, offset, load, area):
        last.update(disp=disp, gap=gap, pressure=pressure, contacting=contacting)
    res = oc.contact_mechanics(h, sizes, periodic=periodic, results_callback=cb, **kw, **opt)
    for key, got in zip(PIPELINE_OUTPUTS, res):
        ref = golden[f"pipe_{name}_{key}"]
        np.testing.assert_allclose(np.asarray(got, dtype=float), ref, rtol=1e-10, atol=1e-14,
                                   err_msg=key)
    for key in ("disp", "gap", "pressure"):
        ref = golden[f"pipe_{name}_last_{key}"]
        np.testing.assert_allclose(last[key], ref, rtol=0, atol=1e-10 * abs(ref).max(), err_msg=key)
    assert np.array_equal(last["contacting"], golden[f"pipe_{name}_last_contacting"])


def test_pipeline_argument_errors():
    """contact_mechanics rejects missing or conflicting step specifications with
    the reference's messages (PipelineFunction.py:314-337), before any solve."""
    import contactmechanics_b200 as cm
    topo = cm.Topography(np.zeros((8, 8)), (1.0, 1.0))
    cases = [(dict(), "Either `nsteps`, `offsets` or `pressures` must be given"),
             (dict(nsteps=2, offsets=[0.1], pressures=[0.1]), "All of"),
             (dict(nsteps=2, offsets=[0.1]), "Both of `nsteps` and `offsets`"),
             (dict(nsteps=2, pressures=[0.1]), "Both of `nsteps` and `pressures`"),
             (dict(offsets=[0.1], pressures=[0.1]), "Both of `offsets` and `pressures`")]
    for kw, msg in cases:
        with pytest.raises(ValueError, match=msg.replace("`", ".")):
            topo.contact_mechanics(**kw)
