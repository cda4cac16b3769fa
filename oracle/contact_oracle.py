"""CPU oracle for the elastic contact solve -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's hot path (ContactEngineering/
ContactMechanics v1.8.3):

* the Green's-function tables and FFT operators of
  ``PeriodicFFTElasticHalfSpace`` and ``FreeFFTElasticHalfSpace``
  (ContactMechanics/FFTElasticHalfSpace.py), and
* the Polonsky-Keer ``constrained_conjugate_gradients`` loop including the
  plastic hardness branches
  (ContactMechanics/Optimization/ConstrainedConjugateGradients.py).

Everything is FP64 / complex128 like the reference.  The reference's FFT
engine (muGrid) is replaced by numpy/scipy pocketfft with the same
conventions: forward transform unnormalised and halved along axis 0, i.e.
``rfftn(a, axes=(1, 0))``.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import this module, and only as the checker or as the timed
CPU baseline.  The product path (``contactmechanics_b200``) never calls it.

Pinning: ``tests/test_oracle.py`` checks this module against golden vectors
produced by running the reference's own code (``tests/golden/make_golden.py``)
and against the reference's analytic known-answer tests.
"""
import math

import numpy as np
import scipy.fft
import scipy.optimize as optim


class SubstrateError(Exception):
    """Mirror of ``Substrate.Error`` (ContactMechanics/Substrates.py:41)."""


class FreeBoundaryError(Exception):
    """Mirror of ``FreeFFTElasticHalfSpace.FreeBoundaryError``
    (ContactMechanics/FFTElasticHalfSpace.py:1207)."""


# ---------------------------------------------------------------------------
# FFT with the reference engine's conventions
# ---------------------------------------------------------------------------

def _axes(ndim):
    return tuple(reversed(range(ndim)))


def fft_forward(a, workers=1):
    """Unnormalised real-to-complex transform, half spectrum along axis 0
    (muGrid convention, FFTElasticHalfSpace.py:104-128)."""
    return scipy.fft.rfftn(a, axes=_axes(a.ndim), workers=workers)


def fft_inverse(fa, shape, workers=1):
    """Unnormalised complex-to-real inverse of :func:`fft_forward`."""
    ax = _axes(len(shape))
    s = [shape[i] for i in ax]
    return scipy.fft.irfftn(fa, s=s, axes=ax, workers=workers) * np.prod(shape)


# ---------------------------------------------------------------------------
# Green's-function tables
# ---------------------------------------------------------------------------

def _wavevectors(n, s):
    """q in cycles per length, ``q = i/s`` for ``i <= n//2`` else ``(n-i)/s``
    (FFTElasticHalfSpace.py:503-515)."""
    i = np.arange(n, dtype=np.float64)
    return np.where(i <= n // 2, i / s, (n - i) / s)


def periodic_greens_function(nb_grid_pts, physical_sizes, young, poisson=0.0,
                             stiffness_q0=None, thickness=None):
    """Periodic table ``G(q) = 1 / (pi E* |q|)`` with the q=0, finite
    thickness and stiffness_q0 variants
    (FFTElasticHalfSpace.py:445-561).  Returns complex128 of shape
    ``(nx//2+1, ny)`` (``(nx//2+1,)`` in 1D)."""
    contact_modulus = young / (1 - poisson ** 2)          # :274
    if len(nb_grid_pts) == 1:                             # :480-499
        (nx,), (sx,) = nb_grid_pts, physical_sizes
        qx = _wavevectors(nx, sx)[:nx // 2 + 1]
        k = np.pi * contact_modulus * qx
        if stiffness_q0 is None:
            k[0] = k[1].real
        elif stiffness_q0 == 0.0:
            k[0] = 1.0
        else:
            k[0] = stiffness_q0
        g = 1 / k
        if stiffness_q0 == 0.0:
            g[0] = 0.0
        return g.astype(complex)
    nx, ny = nb_grid_pts
    sx, sy = physical_sizes
    qx = _wavevectors(nx, sx)[:nx // 2 + 1]
    qy = _wavevectors(ny, sy)
    q = np.sqrt((qx * qx).reshape(-1, 1) + (qy * qy).reshape(1, -1))
    q[0, 0] = np.nan                                      # :516-517
    k = np.pi * contact_modulus * q                       # :521
    if thickness is not None:                             # :524-544
        q = q * (2 * np.pi * thickness)
        fac = 3 - 4 * poisson
        off = 4 * poisson * (2 * poisson - 3) + 5
        with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
            corr = (fac * np.cosh(2 * q) + 2 * q ** 2 + off) / \
                (fac * np.sinh(2 * q) - 2 * q)
        corr[np.isnan(corr)] = 1.0
        k = k * corr
        k[0, 0] = young / thickness * (1 - poisson) / \
            ((1 - 2 * poisson) * (1 + poisson))
    else:                                                 # :546-556
        if stiffness_q0 is None:
            k[0, 0] = (k[1, 0].real + k[0, 1].real) / 2
        elif stiffness_q0 == 0.0:
            k[0, 0] = 1.0
        else:
            k[0, 0] = stiffness_q0
    g = 1 / k                                             # :557
    if stiffness_q0 == 0.0:                               # :558-560
        g[0, 0] = 0.0
    return g.astype(complex)


def surface_stiffness(greens_function):
    """``K = 1/G`` where ``G != 0`` else 0 (FFTElasticHalfSpace.py:563-571)."""
    k = np.zeros(greens_function.shape, dtype=complex)
    nz = greens_function != 0
    k[nz] = 1.0 / greens_function[nz]
    return k


def love_kernel(nb_grid_pts, physical_sizes, young):
    """Real-space displacement of a uniformly loaded ``dx x dy`` pixel on the
    doubled ``(2nx, 2ny)`` domain, coordinates wrapped at ``i > nx``
    (Johnson 1985 p.54; FFTElasticHalfSpace.py:1033-1137)."""
    nx, ny = nb_grid_pts
    dx, dy = physical_sizes[0] / nx, physical_sizes[1] / ny
    a, b = dx / 2, dy / 2
    i = np.arange(2 * nx)
    j = np.arange(2 * ny)
    x = (np.where(i <= nx, i, i - 2 * nx) * dx).reshape(-1, 1)
    y = (np.where(j <= ny, j, j - 2 * ny) * dy).reshape(1, -1)

    def r(p, q):
        return np.sqrt(p * p + q * q)

    xp, xm, yp, ym = x + a, x - a, y + b, y - b
    val = (xp * np.log((yp + r(yp, xp)) / (ym + r(ym, xp)))
           + yp * np.log((xp + r(yp, xp)) / (xm + r(yp, xm)))
           + xm * np.log((ym + r(ym, xm)) / (yp + r(yp, xm)))
           + ym * np.log((xm + r(ym, xm)) / (xp + r(ym, xp))))
    return val / (np.pi * young)


def love_kernel_extended(nb_grid_pts, physical_sizes, young):
    """:func:`love_kernel` evaluated in numpy's extended precision
    (``longdouble``) and rounded once to FP64.  Test helper: the four corner
    terms cancel (by about r^2 at r pixels from the load), so the FP64
    evaluation of the reference formula carries errors of about r^2 eps; the
    extended evaluation measures that error."""
    nx, ny = nb_grid_pts
    L = np.longdouble
    dx, dy = L(physical_sizes[0] / nx), L(physical_sizes[1] / ny)
    a, b = dx / 2, dy / 2
    i = np.arange(2 * nx)
    j = np.arange(2 * ny)
    x = (np.where(i <= nx, i, i - 2 * nx).astype(L) * dx).reshape(-1, 1)
    y = (np.where(j <= ny, j, j - 2 * ny).astype(L) * dy).reshape(1, -1)

    def r(p, q):
        return np.sqrt(p * p + q * q)

    xp, xm, yp, ym = x + a, x - a, y + b, y - b
    val = (xp * np.log((yp + r(yp, xp)) / (ym + r(ym, xp)))
           + yp * np.log((xp + r(yp, xp)) / (xm + r(yp, xm)))
           + xm * np.log((ym + r(ym, xm)) / (yp + r(yp, xm)))
           + ym * np.log((xm + r(ym, xm)) / (xp + r(ym, xp))))
    return (val / (L(np.pi) * L(young))).astype(np.float64)


def _love_at(x, y, dx, dy, young, log=np.log, sqrt=np.sqrt, pi=np.pi):
    """Love's rectangle kernel at offset (x, y) from a uniformly loaded dx x dy
    pixel (the four corner terms of FFTElasticHalfSpace.py:1064-1137)."""
    a, b = dx / 2, dy / 2
    xp, xm, yp, ym = x + a, x - a, y + b, y - b

    def r(p, q):
        return sqrt(p * p + q * q)
    val = (xp * log((yp + r(yp, xp)) / (ym + r(ym, xp)))
           + yp * log((xp + r(yp, xp)) / (xm + r(yp, xm)))
           + xm * log((ym + r(ym, xm)) / (yp + r(yp, xm)))
           + ym * log((xm + r(ym, xm)) / (xp + r(ym, xp))))
    return val / (pi * young)


def semi_periodic_domain(nb_grid_pts, periodicity):
    """Domain of SemiPeriodicFFTElasticHalfSpace: n points along a periodic
    axis, 2n - 1 along a free one (FFTElasticHalfSpace.py:1343-1353)."""
    return tuple(n if per else 2 * n - 1 for n, per in zip(nb_grid_pts, periodicity))


def semi_periodic_kernel(nb_grid_pts, physical_sizes, young, periodicity, n_images,
                         extended=False):
    """Real-space kernel of SemiPeriodicFFTElasticHalfSpace: Love's kernel at
    the signed grid offsets of the domain (numpy fftfreq order, spacing
    L / n), summed over the periodic images -n_images..n_images of each
    periodic axis (FFTElasticHalfSpace.py:1365-1397, 1408-1500).  With
    `extended` the sum is evaluated in numpy's longdouble and rounded once
    (test helper: far images cancel by about r^2 eps in FP64)."""
    nxd, nyd = semi_periodic_domain(nb_grid_pts, periodicity)
    T = np.longdouble if extended else np.float64
    L = [T(v) for v in physical_sizes]
    dx, dy = L[0] / T(nb_grid_pts[0]), L[1] / T(nb_grid_pts[1])
    xs = (np.round(np.fft.fftfreq(nxd) * nxd).astype(T) * dx).reshape(-1, 1)
    ys = (np.round(np.fft.fftfreq(nyd) * nyd).astype(T) * dy).reshape(1, -1)
    imx = range(-n_images, n_images + 1) if periodicity[0] else [0]
    imy = range(-n_images, n_images + 1) if periodicity[1] else [0]
    p = np.zeros((nxd, nyd), dtype=T)
    kw = {}
    if extended:
        kw = dict(pi=T(np.pi) if False else T("3.14159265358979323846264338327950288"))
    for ix in imx:
        for iy in imy:
            p += _love_at(xs + T(ix) * L[0], ys + T(iy) * L[1], dx, dy, T(young), **kw)
    return p.astype(np.float64)


def free_greens_function(nb_grid_pts, physical_sizes, young):
    """Hockney table: forward FFT of :func:`love_kernel`
    (FFTElasticHalfSpace.py:1138-1139).  Shape ``(nx+1, 2ny)`` complex."""
    return fft_forward(love_kernel(nb_grid_pts, physical_sizes, young))


# ---------------------------------------------------------------------------
# Substrates
# ---------------------------------------------------------------------------

class PeriodicSubstrate:
    """Oracle of ``PeriodicFFTElasticHalfSpace`` (FFTElasticHalfSpace.py:151)."""

    is_free = False

    def __init__(self, nb_grid_pts, young, physical_sizes=2 * np.pi,
                 stiffness_q0=None, thickness=None, poisson=0.0, workers=1):
        if not hasattr(nb_grid_pts, "__iter__"):
            nb_grid_pts = (nb_grid_pts,)
        if not hasattr(physical_sizes, "__iter__"):
            physical_sizes = (physical_sizes,)
        self.nb_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self.dim = len(self.nb_grid_pts)
        self.physical_sizes = tuple(
            float(physical_sizes[min(i, len(physical_sizes) - 1)])
            for i in range(self.dim))
        self.young = young
        self.poisson = poisson
        self.contact_modulus = young / (1 - poisson ** 2)
        self.workers = workers
        self.greens_function = periodic_greens_function(
            self.nb_grid_pts, self.physical_sizes, young, poisson,
            stiffness_q0, thickness)
        self.surface_stiffness = surface_stiffness(self.greens_function)

    @property
    def nb_domain_grid_pts(self):
        return self.nb_grid_pts

    @property
    def area_per_pt(self):
        return np.prod(self.physical_sizes) / np.prod(self.nb_grid_pts)

    def _apply(self, table, field, scale):
        n = self.nb_domain_grid_pts
        spec = fft_forward(field, self.workers) * table
        return fft_inverse(spec, n, self.workers) * (scale / np.prod(n))

    def evaluate_disp(self, forces):
        """``u = IFFT(G FFT(-f)) / area_per_pt`` (FFTElasticHalfSpace.py:573-589)."""
        if forces.shape != self.nb_domain_grid_pts:
            raise SubstrateError("force array has a different shape")
        return self._apply(self.greens_function, -forces, 1.0 / self.area_per_pt)

    def evaluate_force(self, disp):
        """``f = -IFFT(K FFT(u)) area_per_pt`` (FFTElasticHalfSpace.py:591-611)."""
        if disp.shape != self.nb_domain_grid_pts:
            raise SubstrateError("displacements array has a different shape")
        return self._apply(self.surface_stiffness, disp, -self.area_per_pt)

    # k-space (FFTElasticHalfSpace.py:613-805): half spectra halved along x
    def evaluate_k_disp(self, forces):
        return self.greens_function * fft_forward(-forces, self.workers) / self.area_per_pt

    def evaluate_k_force(self, disp):
        return -self.surface_stiffness * fft_forward(disp, self.workers) * self.area_per_pt

    def evaluate_k_force_k(self, disp_k):
        return -self.surface_stiffness * disp_k * self.area_per_pt

    def evaluate_scalar_product_k_space(self, ka, kb):
        """Power theorem on rfftn half spectra: rows without a mirror (0 and
        the Nyquist row of an even length) count once, the others twice."""
        nx = self.nb_domain_grid_pts[0]
        w = np.full(ka.shape[0], 2.0)
        w[0] = 1.0
        if nx % 2 == 0:
            w[-1] = 1.0
        prod = (np.conj(ka) * kb).real
        prod = prod.reshape(ka.shape[0], -1)
        return float((w[:, None] * prod).sum() / np.prod(self.nb_domain_grid_pts))

    def evaluate_energy_k(self, disp):
        """``evaluate(disp, pot=True, forces=False)``: the k-space energy."""
        dk = fft_forward(disp, self.workers)
        return -0.5 * self.evaluate_scalar_product_k_space(dk, self.evaluate_k_force_k(dk))


class FreeSubstrate(PeriodicSubstrate):
    """Oracle of ``FreeFFTElasticHalfSpace`` (FFTElasticHalfSpace.py:888)."""

    is_free = True

    def __init__(self, nb_grid_pts, young, physical_sizes=2 * np.pi,
                 check_boundaries=False, workers=1):
        if not hasattr(nb_grid_pts, "__iter__"):
            nb_grid_pts = (nb_grid_pts,)
        if not hasattr(physical_sizes, "__iter__"):
            physical_sizes = (physical_sizes,)
        self.nb_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self.dim = len(self.nb_grid_pts)
        if self.dim != 2:
            raise SubstrateError("free boundaries are implemented for 2D only")
        self.physical_sizes = tuple(
            float(physical_sizes[min(i, len(physical_sizes) - 1)])
            for i in range(self.dim))
        self.young = young
        self.workers = workers
        self.check_boundaries_flag = check_boundaries
        self.greens_function = free_greens_function(
            self.nb_grid_pts, self.physical_sizes, young)
        self.surface_stiffness = surface_stiffness(self.greens_function)

    @property
    def nb_domain_grid_pts(self):
        return tuple(2 * n for n in self.nb_grid_pts)     # :950-951

    def evaluate_disp(self, forces, bIncludePadding=False):
        """Padded input goes straight through; unpadded input is zero-padded
        and only the topography quadrant is returned unless
        ``bIncludePadding`` (FFTElasticHalfSpace.py:1141-1197)."""
        if forces.shape == self.nb_domain_grid_pts:
            return super().evaluate_disp(forces)
        if forces.shape == self.nb_grid_pts:
            padded = np.zeros(self.nb_domain_grid_pts)
            padded[:forces.shape[0], :forces.shape[1]] = forces
            u = super().evaluate_disp(padded)
            if bIncludePadding:
                return u
            return u[:self.nb_grid_pts[0], :self.nb_grid_pts[1]]
        raise SubstrateError("force array has a different shape")

    def check_boundaries(self, force, tol=0):
        """Forces on the outer ring of the topography must vanish
        (FFTElasticHalfSpace.py:1217-1270)."""
        nx, ny = self.nb_grid_pts
        ok = (np.all(abs(force[:, 0]) <= tol) and np.all(abs(force[0, :]) <= tol)
              and np.all(abs(force[:, ny - 1]) <= tol)
              and np.all(abs(force[nx - 1, :]) <= tol))
        if not ok:
            raise FreeBoundaryError(
                "The forces not zero at the boundary of the active domain.")


class SemiPeriodicSubstrate(FreeSubstrate):
    """Oracle of ``SemiPeriodicFFTElasticHalfSpace``
    (FFTElasticHalfSpace.py:1286-1539): free substrate whose periodic axes
    keep n points and sum periodic images into the kernel."""

    def __init__(self, nb_grid_pts, young, physical_sizes=(2 * np.pi, 2 * np.pi),
                 periodicity=(False, True), n_images=10, check_boundaries=False, workers=1,
                 extended=False):
        self.nb_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self.dim = 2
        self.physical_sizes = tuple(float(v) for v in physical_sizes)
        self.young = young
        self.workers = workers
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.n_images = n_images
        self.check_boundaries_flag = check_boundaries
        self.G_real = semi_periodic_kernel(self.nb_grid_pts, self.physical_sizes, young,
                                           self.periodicity, n_images, extended)
        self.greens_function = fft_forward(self.G_real, workers)
        self.surface_stiffness = surface_stiffness(self.greens_function)

    @property
    def nb_domain_grid_pts(self):
        return semi_periodic_domain(self.nb_grid_pts, self.periodicity)

    def evaluate_force(self, disp):
        """Displacements that do not cover the domain are zero padded
        (FFTElasticHalfSpace.py:1541-1565)."""
        if disp.shape != self.nb_domain_grid_pts:
            padded = np.zeros(self.nb_domain_grid_pts)
            padded[:disp.shape[0], :disp.shape[1]] = disp
            disp = padded
        return super().evaluate_force(disp)


# ---------------------------------------------------------------------------
# Polonsky-Keer constrained conjugate gradients
# ---------------------------------------------------------------------------

def rms_height(heights):
    """rms height about the mean (used for the default ``pentol``)."""
    h = np.asarray(heights)
    return float(np.sqrt(np.mean((h - h.mean()) ** 2)))


def constrained_conjugate_gradients(substrate, heights, hardness=None,
                                    external_force=None, offset=None,
                                    initial_displacements=None,
                                    initial_forces=None, pentol=None,
                                    forcetol=1e-5, thermotol=1e-6,
                                    mixfac=0.1, mixdecfac=0.95,
                                    minmixsteps=10, maxiter=100000,
                                    callback=None):
    """Restatement of ``constrained_conjugate_gradients``
    (ConstrainedConjugateGradients.py:47-509), serial, unmasked heights.

    Returns a dict with the fields of the reference's ``OptimizeResult``.
    """
    heights = np.asarray(heights, dtype=np.float64)
    nb_surface_pts = heights.size
    if pentol is None:                                    # :150-162
        pentol = rms_height(heights) / (10 * np.mean(heights.shape))
        if pentol == 0:
            pentol = ((offset if offset is not None else 0)
                      + heights.sum() / nb_surface_pts) / 1000
        if pentol == 0:
            pentol = 1e-3
    if offset is None:
        offset = 0
    dom = substrate.nb_domain_grid_pts
    if initial_displacements is None:
        u_r = np.zeros(dom)
    else:
        u_r = np.array(initial_displacements, dtype=np.float64, copy=True)
    comp_slice = tuple(slice(0, n) for n in substrate.nb_grid_pts)   # :179-181
    comp_mask = np.zeros(dom, dtype=bool)
    comp_mask[comp_slice] = True
    masked_surface = heights.ravel()                      # :189-194 (no mask)
    max_masked_surface = masked_surface.max()
    pad_mask = ~comp_mask
    n_pad = int(pad_mask.sum())
    lo = masked_surface + offset                          # :201
    uc = u_r[comp_mask]
    u_r[comp_mask] = np.where(uc < lo, lo, uc)

    nfev = 0
    if initial_forces is None:                            # :211-215
        f_r = substrate.evaluate_force(u_r)
    else:
        f_r = np.array(initial_forces, dtype=np.float64, copy=True)
        u_r = substrate.evaluate_disp(f_r)
    nfev += 1
    f_r[pad_mask] = 0.0                                   # :219

    delta, delta_str, G_old = 0, "reset", 1.0             # :222-224
    t_r = np.zeros_like(u_r)
    tau = 0.0
    current_mixfac, mixsteps = mixfac, 0
    last_max_height = last_total_force = None
    A_fl = 0
    result = dict(success=False, message="Not Converged (yet)")

    for it in range(1, maxiter + 1):
        c_r = f_r < 0.0                                   # :239
        A_contact = int(c_r.sum())
        if hardness is not None:                          # :247-249
            c_r = np.logical_and(c_r, f_r > -hardness)
        A_cg = int(c_r.sum())
        if hardness is None or (A_contact > 0 and A_cg / A_contact > 0.01
                                and mixsteps <= 0):       # :260
            if delta_str == "mix":
                delta_str = "sd"
            g_r = u_r[comp_mask] - masked_surface         # :265
            if external_force is not None:
                offset = 0
                if A_cg > 0:
                    offset = g_r[c_r[comp_mask]].sum() / A_cg
            g_r -= offset
            G = (c_r[comp_mask] * g_r * g_r).sum()        # :273
            if delta > 0 and G_old > 0:                   # :276-279
                t_r[comp_mask] = c_r[comp_mask] * (g_r + delta * (G / G_old) * t_r[comp_mask])
            else:
                t_r[comp_mask] = c_r[comp_mask] * g_r
            r_r = substrate.evaluate_disp(t_r)            # :284
            nfev += 1
            tau = 0.0
            if A_cg > 0:                                  # :287-294
                x = -(c_r * r_r * t_r).sum()
                if x > 0.0:
                    tau = (c_r[comp_mask] * g_r * t_r[comp_mask]).sum() / x
                else:
                    G = 0.0
            f_r += tau * c_r * t_r                        # :296
            current_mixfac = mixfac
        else:                                             # :300-330
            if delta_str != "mix":
                mixsteps = minmixsteps
                delta_str = "mix"
            g_r = u_r[comp_mask] - masked_surface
            if external_force is not None:
                gg = g_r
                offset = optim.bisect(
                    lambda x: ((gg - x) < 0.0).sum() * hardness - external_force,
                    gg.max(), gg.min())
            g_r -= offset
            c_r[comp_mask] = g_r < 0.0
            f_r = (1 - current_mixfac) * f_r - current_mixfac * hardness * c_r
            current_mixfac *= mixdecfac
            if mixsteps > 0:
                mixsteps -= 1
        mask_tensile = f_r >= 0.0                         # :334
        nc_r = np.logical_and(mask_tensile[comp_mask], g_r < 0.0)
        if hardness is not None:                          # :338-340
            mask_flowing = f_r <= -hardness
            nc_r = np.logical_or(nc_r, np.logical_and(mask_flowing[comp_mask], g_r > 0.0))
        pad_pres = 0                                      # :344-346
        if n_pad > 0:
            pad_pres = abs(f_r[pad_mask]).max()
        max_pres = 0                                      # :350-356
        if mask_tensile.sum() > 0:
            max_pres = (f_r[mask_tensile] * 1).max()
        if hardness:
            A_fl = int(mask_flowing.sum())
            if A_fl > 0:
                max_pres = max(max_pres, -(f_r[mask_flowing] + hardness).min())
        f_r[mask_tensile] = 0.0                           # :359
        if external_force is not None:                    # :362-368
            total_force = -f_r[comp_mask].sum()
            if total_force != 0:
                f_r *= external_force / total_force
            else:
                f_r = -external_force / nb_surface_pts * np.ones_like(f_r)
                f_r[pad_mask] = 0.0
        if hardness is not None:                          # :372-373
            f_r[mask_flowing] = -hardness
        if delta_str == "mix":                            # :375-389
            delta = 0
            G = 0
        else:
            if nc_r.sum() > 0:
                f_r[comp_mask] += tau * nc_r * g_r
                delta = 0
                delta_str = "sd"
            else:
                delta = 1
                delta_str = "cg"
        new_u_r = substrate.evaluate_disp(f_r)            # :393
        maxdu = abs(new_u_r - u_r).max()
        u_r = new_u_r
        nfev += 1
        G_old = G
        rms_pen = math.sqrt(G / A_cg) if A_cg > 0 else math.sqrt(G)   # :403-406
        max_pen = max(0.0, (c_r[comp_mask] * (masked_surface + offset - u_r[comp_mask])).max())
        converged = True                                  # :414-434
        total_force = -f_r[comp_mask].sum()
        if external_force is not None:
            converged = converged and abs((total_force - external_force) / total_force) < thermotol
        elif last_total_force is not None:
            converged = converged and abs((total_force - last_total_force) / total_force) < thermotol
        last_total_force = total_force
        max_height = max_masked_surface + offset
        if external_force is not None and last_max_height is not None:
            converged = converged and abs((max_height - last_max_height) / max_height) < thermotol
        last_max_height = max_height
        if delta_str == "mix":
            converged = converged and maxdu < pentol and max_pres < forcetol and pad_pres < forcetol
        else:
            converged = (converged and rms_pen < pentol and max_pen < pentol and maxdu < pentol
                         and max_pres < forcetol and pad_pres < forcetol)
        result.update(nit=it, nfev=nfev, maxcv=dict(max_pen=max_pen, max_pres=max_pres))
        if converged:                                     # :454-475
            result["x"] = u_r
            result["jac"] = -f_r[comp_slice]
            result["active_set"] = c_r.copy()
            if hardness is not None:
                plastic = np.zeros_like(c_r)
                plastic[comp_mask] = g_r < 0.0
                result["plastic"] = plastic[comp_slice]
            if delta_str == "mix":
                result["active_set"][comp_mask] = g_r < 0.0
            result["fun"] = -(f_r[comp_slice] * u_r[comp_slice]).sum() / 2
            result["offset"] = offset
            result["success"] = True
            result["message"] = "Polonsky converged"
            return result
        if callback is not None:
            callback(it, f_r, dict(area=A_contact, rms_penetration=rms_pen,
                                   max_penetration=max_pen, max_pressure=max_pres,
                                   pad_pressure=pad_pres))
        if math.isnan(G) or math.isnan(rms_pen):          # :491-492
            raise RuntimeError("nan encountered.")
    result["x"] = u_r                                     # :494-509
    result["jac"] = -f_r[comp_slice]
    result["active_set"] = c_r
    result["fun"] = -(f_r[comp_slice] * u_r[comp_slice]).sum() / 2
    result["offset"] = offset
    result["message"] = "Reached maxiter = {}".format(maxiter)
    return result


# ---------------------------------------------------------------------------
# Seeded synthetic inputs (shared by tests and the CPU baseline)
# ---------------------------------------------------------------------------

def sphere(nb_grid_pts, physical_sizes, radius=1.0):
    """Paraboloid ``h = -r^2/(2R)`` centred at ``(n/2) dx``."""
    nx, ny = nb_grid_pts
    sx, sy = physical_sizes
    x = ((np.arange(nx) - nx / 2) * sx / nx).reshape(-1, 1)
    y = ((np.arange(ny) - ny / 2) * sy / ny).reshape(1, -1)
    return -(x * x + y * y) / (2 * radius)


def self_affine(nb_grid_pts, physical_sizes, hurst, rms_slope, seed,
                short_cutoff_px=4.0, rolloff_wavelength=None):
    """Seeded Gaussian self-affine surface: isotropic PSD ``C(q) ~ q^-2(1+H)``
    above the rolloff wavevector (flat below it), zero above the short
    wavelength cutoff, ``C(0) = 0``; rescaled to the requested rms slope."""
    nx, ny = nb_grid_pts
    sx, sy = physical_sizes
    rng = np.random.default_rng(seed)
    qx = 2 * np.pi * np.fft.fftfreq(nx, d=sx / nx).reshape(-1, 1)
    qy = 2 * np.pi * np.fft.rfftfreq(ny, d=sy / ny).reshape(1, -1)
    q = np.sqrt(qx * qx + qy * qy)
    if rolloff_wavelength is None:
        rolloff_wavelength = max(sx, sy) / 8
    q_r = 2 * np.pi / rolloff_wavelength
    q_s = 2 * np.pi / (short_cutoff_px * max(sx / nx, sy / ny))
    qq = np.maximum(q, q_r)
    amp = qq ** (-(1 + hurst))
    amp[q > q_s] = 0
    amp[0, 0] = 0
    phase = np.exp(2j * np.pi * rng.random(amp.shape))
    noise = rng.standard_normal(amp.shape)
    h = np.fft.irfft2(amp * noise * phase, s=(nx, ny))
    dx = np.diff(h, axis=0, append=h[:1, :]) / (sx / nx)
    dy = np.diff(h, axis=1, append=h[:, :1]) / (sy / ny)
    slope = np.sqrt(np.mean(dx * dx + dy * dy))
    return h * (rms_slope / slope)


# ---------------------------------------------------------------------------
# Automated sweeps (PipelineFunction.py:37-449)
# ---------------------------------------------------------------------------

def auto_offset(step, mean_displacements, total_contact_areas, heights):
    """Offset of automatic step `step` of a sweep from the offsets and contact
    areas of the steps before it (PipelineFunction.py:138-226)."""
    top, middle, bot = np.max(heights), np.mean(heights), np.min(heights)
    if step == 0:
        return -middle
    if step == 1:
        return -top + 0.01 * (top - middle)
    sd, sa = np.transpose(sorted(zip(mean_displacements, total_contact_areas),
                                 key=lambda pair: pair[1]))
    ref_area = np.log10(np.array(sa + 1 / np.prod(np.shape(heights))))
    darea = np.append(ref_area[1:] - ref_area[:-1], -ref_area[-1])
    i = np.argmax(darea)
    return bot + 2 * (sd[-1] - bot) if i == step - 1 else (sd[i] + sd[i + 1]) / 2


def contact_mechanics(heights, physical_sizes, periodic=True, nsteps=None, offsets=None,
                      pressures=None, hardness=None, maxiter=100, results_callback=None,
                      **solver_kwargs):
    """Restatement of ``contact_mechanics`` (PipelineFunction.py:229-449) with
    this module's solver.  A hardness (units of E*) makes it plastic: the
    solver gets ``hardness * area_per_pt`` and, after each converged solve,
    the plastic gap is added to the plastic displacement
    (PlasticSystemSpecialisations.py:60-69); automatically chosen steps reset
    it first (PipelineFunction.py:171-178).  Returns mean pressure, contact
    area, mean displacement, mean gap and convergence flags per step."""
    h0 = np.asarray(heights, dtype=np.float64)
    nb = h0.shape
    sub = (PeriodicSubstrate if periodic else FreeSubstrate)(nb, 1.0, physical_sizes)
    plastic = hardness is not None and hardness > 0
    state = {"pd": np.zeros(nb)}

    def cur_heights():
        return h0 + state["pd"] if plastic else h0

    # pentol from the rms height (PipelineFunction.py:390-393)
    pentol = max(rms_height(h0 + state["pd"] if plastic else h0) / (10 * np.mean(nb)), 1e-12)
    md, mg, mp, ta, conv = [], [], [], [], []

    def calc(offset=None, external_force=None):
        middle = np.mean(cur_heights())
        kw = dict(solver_kwargs)
        if plastic:
            kw["hardness"] = hardness * sub.area_per_pt
        r = constrained_conjugate_gradients(sub, cur_heights(), offset=offset,
                                            external_force=external_force, pentol=pentol,
                                            maxiter=maxiter, **kw)
        force = r["jac"]
        disp = r["x"][:force.shape[0], :force.shape[1]]
        if plastic and r["success"]:
            gap = disp - (cur_heights() + r["offset"])
            state["pd"] = state["pd"] + np.where(r["plastic"], gap, 0.0)
        md.append(r["offset"])
        mg.append(np.mean(disp) - middle - r["offset"])
        load = force.sum() / np.prod(physical_sizes)
        mp.append(load)
        area = (force > 0).sum() / np.prod(nb)
        ta.append(area)
        conv.append(bool(r["success"]))
        if results_callback is not None:
            gap_xy = disp - cur_heights() - r["offset"]
            gap_xy[gap_xy < 0.0] = 0.0
            results_callback(disp, gap_xy, force / sub.area_per_pt, force > 0, r["offset"], load,
                             area)

    if pressures is not None:
        for p in pressures:
            calc(external_force=p * np.prod(physical_sizes))
    elif offsets is not None:
        for o in offsets:
            calc(offset=o)
    else:
        for step in range(nsteps):
            state["pd"] = np.zeros(nb)
            calc(offset=auto_offset(step, md, ta, cur_heights()))
    return np.array(mp), np.array(ta), np.array(md), np.array(mg), np.array(conv)

