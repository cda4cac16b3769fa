"""The periodic operator entry point that allocates nothing.

``cm_apply_periodic_noalloc`` serves callers that must not allocate device
memory themselves or through the library -- for example a host application
that hands out all device memory from its own pool, or a time-critical loop
that cannot risk the device-wide synchronisation a cudaMalloc may cause.  It
keeps its Green's table, twiddles and spectrum in a fixed array inside the
library, so it needs no plan.  This test calls it through the C ABI twice in
a row for two grids (the second call reuses the scratch the first one left
behind) and compares each result with the plan-based operator (cm_apply via
the substrate classes) within the FP64 operator tolerance used by the other
tests: 1e-12 of the field's largest magnitude.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = [
    # grid, physical sizes, Young's modulus, Poisson ratio, operator
    ((64, 48), (1.3, 0.7), 1.1, 0.3, "disp"),
    ((96, 128), (2.0, 1.0), 2.5, 0.0, "force"),
    ((512, 500), (1.0, 1.0), 1.0, 0.0, "disp"),
]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_operator_matches_plan_operator_on_repeated_calls():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    from contactmechanics_b200 import _lib

    L = _lib.lib()
    gen = torch.Generator(device="cuda").manual_seed(7)
    for call in range(2):
        for nb, sizes, young, poisson, op in CASES:
            field = torch.randn(nb, dtype=torch.float64, device="cuda", generator=gen)
            out = torch.empty_like(field)
            code = _lib.CM_OP_DISP if op == "disp" else _lib.CM_OP_FORCE
            rc = L.cm_apply_periodic_noalloc(nb[0], nb[1], sizes[0], sizes[1], young, poisson,
                                             code, _ptr(field), _ptr(out), None)
            assert rc == _lib.CM_OK, _lib.status_string(rc)
            torch.cuda.synchronize()
            sub = cm.PeriodicFFTElasticHalfSpace(nb, young, sizes, poisson=poisson)
            ref = sub.evaluate_disp(field) if op == "disp" else sub.evaluate_force(field)
            ref = ref.cpu().numpy()
            np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0,
                                       atol=1e-12 * np.abs(ref).max(),
                                       err_msg=f"call {call}, grid {nb}, {op}")


def test_noalloc_operator_rejects_grids_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from contactmechanics_b200 import _lib

    L = _lib.lib()
    field = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    rc = L.cm_apply_periodic_noalloc(1024, 1024, 1.0, 1.0, 1.0, 0.0, _lib.CM_OP_DISP,
                                     _ptr(field), _ptr(field), None)
    assert rc == _lib.CM_ERR_SIZE
