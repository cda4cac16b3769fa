"""Plastic mixed-precision solves whose FP32 phase stalls (GPU)."""
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


# Plastic loads whose FP32 phase stalls at FP32 resolution (seeded surfaces
# and loads of the serving benchmark's request stream): the FP64 oracle
# solves them in 25 and 214 iterations; the mixed solve must hand its FP32
# phase over within the plastic cap and agree with the oracle.
PLASTIC_STALL_CASES = [
    # (kind, side, surface index, load F, hardness per point)
    ("periodic", 96, 4, 1.7772509896851914e-4, 9.850516127608379e-6),
    ("free", 128, 5, 9.582191995047694e-3, 1.362818710820602e-6),
]


@pytest.mark.parametrize("kind,side,k,F,H", PLASTIC_STALL_CASES)
def test_plastic_mixed_fp32_phase_is_capped(cm, kind, side, k, F, H):
    from contactmechanics_b200.Generation import self_affine
    h = self_affine((side, side), (1.0, 1.0), 0.8, 0.1, seed=1000 * side + k)
    kw = dict(external_force=F, hardness=H, pentol=1e-9 * float(h.max() - h.min()),
              forcetol=1e-9 * F, maxiter=20000)
    cls = cm.FreeFFTElasticHalfSpace if kind == "free" else cm.PeriodicFFTElasticHalfSpace
    res = cm.constrained_conjugate_gradients(cls((side, side), 1.0, (1.0, 1.0)), h,
                                             precision="mixed", **kw)
    assert res.success
    # the FP32 phase ran to the plastic cap without converging, and the FP64
    # refinement that followed finished the solve within maxiter
    assert res.nit_fp32 == 256, res.nit_fp32
    assert res.nit <= kw["maxiter"]
    assert res.nit > res.nit_fp32
    ocls = oc.FreeSubstrate if kind == "free" else oc.PeriodicSubstrate
    ref = oc.constrained_conjugate_gradients(ocls((side, side), 1.0, (1.0, 1.0)), h, **kw)
    assert ref["success"]
    x = ref["x"][:side, :side]
    rel = np.linalg.norm(res.x[:side, :side] - x) / np.linalg.norm(x)
    assert rel <= 1e-6, rel
