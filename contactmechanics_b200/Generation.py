"""Seeded synthetic topographies (host-side input generation).

``sphere`` is the paraboloid ``h = -r^2/(2R)`` centred at ``(n/2) dx`` used
for Hertzian contact.  ``self_affine`` is a Gaussian random rough surface
with isotropic power spectrum ``C(q) ~ q^-2(1+H)`` above a rolloff
wavevector (flat below it), zero above a short-wavelength cutoff and at
q = 0, rescaled to a target rms slope.  They stand in for SurfaceTopography's
generators, which are not part of this package.
"""
import numpy as np


def sphere(nb_grid_pts, physical_sizes, radius=1.0):
    nx, ny = nb_grid_pts
    sx, sy = physical_sizes
    x = ((np.arange(nx) - nx / 2) * sx / nx).reshape(-1, 1)
    y = ((np.arange(ny) - ny / 2) * sy / ny).reshape(1, -1)
    return -(x * x + y * y) / (2 * radius)


def self_affine(nb_grid_pts, physical_sizes, hurst, rms_slope, seed, short_cutoff_px=4.0,
                rolloff_wavelength=None):
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
    amp = np.maximum(q, q_r) ** (-(1 + hurst))
    amp[q > q_s] = 0
    amp[0, 0] = 0
    phase = np.exp(2j * np.pi * rng.random(amp.shape))
    noise = rng.standard_normal(amp.shape)
    h = np.fft.irfft2(amp * noise * phase, s=(nx, ny))
    dx = np.diff(h, axis=0, append=h[:1, :]) / (sx / nx)
    dy = np.diff(h, axis=1, append=h[:, :1]) / (sy / ny)
    slope = np.sqrt(np.mean(dx * dx + dy * dy))
    return h * (rms_slope / slope)
