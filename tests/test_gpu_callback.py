"""Per-iteration callback and logger (ConstrainedConjugateGradients.py
:436-489) against the oracle, which calls its callback exactly where the
reference does: after every iteration that did not converge, with the
iteration's forces on the domain and the scalar record d.
"""
import io

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


def _record(store):
    def cb(it, f, d):
        f = f.detach().cpu().numpy() if hasattr(f, "detach") else np.asarray(f)
        store.append((it, f.copy(), dict(d)))
    return cb


@pytest.mark.parametrize("kind,hardness", [("periodic", None), ("free", None), ("periodic", 0.05)])
def test_callback_sequence_matches_oracle(cm, kind, hardness):
    nb = (64, 64)
    if kind == "periodic":
        h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=11)
        sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
        o = oc.PeriodicSubstrate(nb, 1.0, (1.0, 1.0))
    else:
        h = oc.sphere(nb, (1.0, 1.0), 2.0)
        sub = cm.FreeFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
        o = oc.FreeSubstrate(nb, 1.0, (1.0, 1.0))
    kw = dict(external_force=2e-3, pentol=1e-10 * float(h.max() - h.min()), forcetol=1e-12)
    if hardness is not None:
        kw["hardness"] = hardness * o.area_per_pt
        kw["forcetol"] = 1e-10
    ours, ref = [], []
    res = cm.constrained_conjugate_gradients(sub, h, precision="fp64", callback=_record(ours), **kw)
    rr = oc.constrained_conjugate_gradients(o, h, callback=_record(ref), **kw)
    assert res.success and rr["success"]
    # one record per iteration that did not converge, numbered 1 .. nit-1
    assert [r[0] for r in ours] == [r[0] for r in ref] == list(range(1, res.nit))
    for (it, f, d), (_, fr, dr) in zip(ours, ref):
        assert f.shape == fr.shape == tuple(sub.nb_domain_grid_pts)
        scale = max(abs(fr).max(), 1e-300)
        np.testing.assert_allclose(f, fr, rtol=0, atol=1e-9 * scale, err_msg=f"it {it}")
        assert d["area"] == dr["area"], it
        for key in ("rms_penetration", "max_penetration", "max_pressure", "pad_pressure"):
            np.testing.assert_allclose(d[key], dr[key], rtol=1e-7, atol=1e-14, err_msg=key)
        assert d["penetration_tol"] == pytest.approx(kw["pentol"])
        assert d["pressure_tol"] == kw["forcetol"]


def test_callback_mixed_counts_through_both_phases(cm):
    nb = (64, 64)
    h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=12)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    seen = []
    res = cm.constrained_conjugate_gradients(sub, h, external_force=2e-3, precision="mixed",
                                             pentol=1e-9 * float(h.max() - h.min()),
                                             forcetol=1e-12,
                                             callback=lambda it, f, d: seen.append(it))
    assert res.success and res.nit_fp32 > 0
    # every iteration of both phases except the converged last one
    assert len(seen) >= res.nit - 2 and seen == sorted(seen)
    assert seen[-1] >= res.nit_fp32


def test_callback_exception_stops_the_solve(cm):
    nb = (64, 64)
    h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=13)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    calls = []

    def cb(it, f, d):
        calls.append(it)
        if it == 3:
            raise KeyboardInterrupt("stop")

    with pytest.raises(KeyboardInterrupt):
        cm.constrained_conjugate_gradients(sub, h, external_force=2e-3, precision="fp64",
                                           pentol=1e-10 * float(h.max() - h.min()),
                                           forcetol=1e-12, callback=cb)
    assert calls == [1, 2, 3]
    # the plan stays usable
    res = cm.constrained_conjugate_gradients(sub, h, external_force=2e-3, precision="fp64")
    assert res.success


def test_logger_rows_per_iteration(cm):
    from contactmechanics_b200.Tools.Logger import Logger
    nb = (64, 64)
    h = oc.self_affine(nb, (1.0, 1.0), 0.8, 0.1, seed=14)
    sub = cm.PeriodicFFTElasticHalfSpace(nb, 1.0, (1.0, 1.0))
    buf = io.StringIO()
    res = cm.constrained_conjugate_gradients(sub, h, external_force=2e-3, precision="fp64",
                                             pentol=1e-10 * float(h.max() - h.min()),
                                             forcetol=1e-12, logger=Logger(buf), verbose=True)
    assert res.success
    rows = [line for line in buf.getvalue().splitlines() if line.startswith(" ")]
    # one row per iteration that did not converge, then the final CONVERGED row
    assert len(rows) == res.nit
    assert rows[-1].split()[0] == "CONVERGED"
    assert rows[0].split()[0] in ("sd", "cg") and rows[0].split()[1] == "1"
