"""Domains of 8192 points per side (GPU): the power-of-two passes at 2^13,
where FP64 transforms run on one shared-memory buffer with global
twiddles.  A free 4096^2 topography (the largest free request of the
serving workload) has such a domain.

* periodic 8192^2 operator against the oracle (FP64 to 1e-12, FP32 to 2e-5
  of the field maximum);
* free 4096^2 operator (8192^2 domain) against the oracle: the reference's
  Love-kernel formula evaluated in FP64 cancels by about r^2 eps at r
  pixels, an error that grows with the square of the grid (2e-9 of the
  field in 2-norm at 1024^2, 5e-8 in max-norm at 4096^2); the library
  evaluates it in extended precision, so the FP64 operators agree to 1e-7
  of the field maximum, and the library's kernel (the inverse transform of
  its table) matches the kernel evaluated in long double at sampled offsets,
  far ones included, to 1e-12; FP32 against FP64 to 2e-5;
* a free 4096^2 contact solve: mixed precision within 1e-6 (displacement)
  and 1e-3 (contact area) of the FP64 solve, both meeting the load.
"""
import os

import numpy as np
import pytest

from oracle import contact_oracle as oc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
WORKERS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def cm():
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import contactmechanics_b200 as cm
    return cm


def test_periodic_8192_operator(cm):
    n = 8192
    rng = np.random.default_rng(81)
    f = rng.standard_normal((n, n))
    o = oc.PeriodicSubstrate((n, n), 1.0, (1.0, 1.0), workers=WORKERS)
    ref = o.evaluate_disp(f)
    for prec, tol in (("fp64", 1e-12), ("fp32", 2e-5)):
        s = cm.PeriodicFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0), precision=prec)
        got = s.evaluate_disp(torch.from_numpy(f).cuda()).cpu().numpy()
        err = abs(got - ref).max() / abs(ref).max()
        assert err < tol, (prec, err)


def test_free_4096_operator(cm):
    n = 4096
    rng = np.random.default_rng(82)
    f = rng.standard_normal((n, n))
    o = oc.FreeSubstrate((n, n), 1.0, (1.0, 1.0), workers=WORKERS)
    ref = o.evaluate_disp(f, bIncludePadding=True)
    s = cm.FreeFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
    assert s.nb_domain_grid_pts == (2 * n, 2 * n)
    fd = torch.from_numpy(f).cuda()
    got = s.evaluate_disp(fd, bIncludePadding=True).cpu().numpy()
    assert abs(got - ref).max() / abs(ref).max() < 1e-7
    s32 = cm.FreeFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0), precision="fp32")
    got32 = s32.evaluate_disp(fd, bIncludePadding=True).cpu().numpy()
    assert abs(got32 - got).max() / abs(got).max() < 2e-5
    # the library's table is the transform of the exactly evaluated kernel:
    # its inverse transform matches the kernel evaluated in long double at
    # sampled offsets, the far ones included
    nd = 2 * n
    kern = np.fft.irfftn(s.greens_function, s=(nd, nd), axes=(1, 0))
    L = np.longdouble
    dx = L(1) / L(n)
    idx = np.concatenate([rng.integers(0, nd, (400, 2)),
                          [[n, n], [n - 1, n], [n, 0], [0, n], [1, 1], [0, 0]]])
    for i, j in idx:
        si = i if i <= n else i - nd
        sj = j if j <= n else j - nd
        exact = float(oc._love_at(L(si) * dx, L(sj) * dx, dx, dx, L(1.0),
                                  pi=L("3.14159265358979323846264338327950288")))
        assert abs(kern[i, j] - exact) <= 1e-12 * abs(kern).max(), (i, j, kern[i, j], exact)


def test_free_4096_solve_mixed_vs_fp64(cm):
    from contactmechanics_b200.Generation import self_affine
    n = 4096
    h = self_affine((n, n), (1.0, 1.0), 0.8, 0.1, seed=4096)
    F = 1e-3
    kw = dict(external_force=F, pentol=1e-9 * float(h.max() - h.min()), forcetol=1e-12 * F)
    s = cm.FreeFFTElasticHalfSpace((n, n), 1.0, (1.0, 1.0))
    hd = torch.from_numpy(h).cuda()
    r64 = cm.constrained_conjugate_gradients(s, hd, precision="fp64", **kw)
    rmx = cm.constrained_conjugate_gradients(s, hd, precision="mixed", **kw)
    assert r64.success and rmx.success
    x64, xmx = r64.x[:n, :n], rmx.x[:n, :n]
    assert float(torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64)) < 1e-6
    a64, amx = int((r64.jac > 0).sum()), int((rmx.jac > 0).sum())
    assert abs(amx - a64) <= 1e-3 * a64
    for r in (r64, rmx):
        np.testing.assert_allclose(float(r.jac.sum()), F, rtol=1e-6)
