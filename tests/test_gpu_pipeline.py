"""The automated sweep (contact_mechanics) on the device solver against the
reference's own sweeps: per-step mean pressures, contact areas, mean
displacements and gaps and convergence flags, and the last step's fields,
for listed pressures, automatically chosen offsets (free boundaries) and
listed offsets with plastic history.  FP64 to 1e-10; mixed precision to 1e-6
(relative, per-step means) and 1e-3 (contact areas)."""
import numpy as np
import pytest

from tests.conftest import GOLDEN, PIPELINE_OUTPUTS, golden_pipeline_case, golden_pipeline_names

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

_npz = np.load(GOLDEN)


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def _run(cm, golden, name, precision):
    h, sizes, periodic, kw = golden_pipeline_case(golden, name)
    kw["optimizer_kwargs"] = dict(kw.get("optimizer_kwargs", {}), precision=precision)
    last = {}

    def cb(disp, gap, pressure, contacting, offset, load, area):
        last.update(disp=disp, gap=gap, pressure=pressure, contacting=contacting)
    topo = cm.Topography(h, sizes, periodic=periodic)
    return topo.contact_mechanics(results_callback=cb, **kw), last


@pytest.mark.parametrize("name", golden_pipeline_names(_npz))
def test_pipeline_fp64_vs_reference(cm, golden, name):
    res, last = _run(cm, golden, name, "fp64")
    for key, got in zip(PIPELINE_OUTPUTS, res):
        ref = golden[f"pipe_{name}_{key}"]
        np.testing.assert_allclose(np.asarray(got, dtype=float), ref, rtol=1e-10, atol=1e-14,
                                   err_msg=key)
    for key in ("disp", "gap", "pressure"):
        ref = golden[f"pipe_{name}_last_{key}"]
        np.testing.assert_allclose(last[key], ref, rtol=0, atol=1e-10 * abs(ref).max(), err_msg=key)
    assert np.array_equal(last["contacting"], golden[f"pipe_{name}_last_contacting"])


@pytest.mark.parametrize("name", golden_pipeline_names(_npz))
def test_pipeline_mixed_vs_reference(cm, golden, name):
    """The sweep picks its own, loose penetration tolerance
    pentol = rms height / (10 mean(n)); a mixed solve stops at another point
    of that tolerance than the reference's FP64 path, so offsets and gaps are
    compared to 2 pentol, mean pressures to 1e-3 relative (plus the same
    pentol-sized slack in offset control), contact areas to 1e-3."""
    h, *_ = golden_pipeline_case(golden, name)
    pentol = max(np.sqrt(np.mean((h - h.mean()) ** 2)) / (10 * np.mean(h.shape)), 1e-12)
    res, _ = _run(cm, golden, name, "mixed")
    got = dict(zip(PIPELINE_OUTPUTS, res))
    assert np.array_equal(got["converged"], golden[f"pipe_{name}_converged"])
    for key in ("mean_displacement", "mean_gap"):
        ref = golden[f"pipe_{name}_{key}"]
        np.testing.assert_allclose(got[key], ref, rtol=0, atol=2 * pentol, err_msg=key)
    ref = golden[f"pipe_{name}_mean_pressure"]
    np.testing.assert_allclose(got["mean_pressure"], ref, rtol=1e-3, atol=2 * pentol,
                               err_msg="mean_pressure")
    ref = golden[f"pipe_{name}_area"]
    np.testing.assert_allclose(got["area"], ref, rtol=1e-3, err_msg="area")
