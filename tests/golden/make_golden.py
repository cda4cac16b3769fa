"""Generate golden vectors by running the reference's own code.

Run where a checkout of the reference is available (read-only is enough)::

    python tests/golden/make_golden.py /path/to/reference [--only=main|semi|kspace]
    # or: CM_REFERENCE=/path/to/reference python tests/golden/make_golden.py

It imports ContactMechanics unmodified over the serial stand-ins of
``refstubs.py`` and writes ``tests/golden/reference_vectors.npz`` (operators,
solves, sweeps), ``semi_vectors.npz`` (SemiPeriodicFFTElasticHalfSpace) and
``kspace_vectors.npz`` (k-space operators and energies); ``--only=`` picks
one of them.  The fixtures are small
(grids of at most 64x64) so that the CPU test-suite stays fast.  The GPU box
never runs this script; tests only read the committed ``.npz`` files.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import refstubs  # noqa: E402


def _sphere(nb, sizes, radius):
    nx, ny = nb
    sx, sy = sizes
    x = ((np.arange(nx) - nx / 2) * sx / nx).reshape(-1, 1)
    y = ((np.arange(ny) - ny / 2) * sy / ny).reshape(1, -1)
    return -(x * x + y * y) / (2 * radius)


def main(ref_root):
    refstubs.install(ref_root)
    from ContactMechanics import (PeriodicFFTElasticHalfSpace,
                                  FreeFFTElasticHalfSpace)
    from ContactMechanics.Systems import NonSmoothContactSystem
    from ContactMechanics.PlasticSystemSpecialisations import \
        PlasticNonSmoothContactSystem
    from oracle.contact_oracle import self_affine

    rng = np.random.default_rng(20261203)
    out = {}

    # ---- operators --------------------------------------------------------
    periodic_cases = [
        ("p8x15", (8, 15), (2.45, 1.0), {}),
        ("p9x4", (9, 4), (2.45, 1.0), {}),
        ("p16x16_q0zero", (16, 16), (1.0, 1.0), dict(stiffness_q0=0.0)),
        ("p16x12_q0val", (16, 12), (3.0, 2.0), dict(stiffness_q0=2.5)),
        ("p32x24_thick", (32, 24), (1.0, 1.5), dict(thickness=0.2, poisson=0.3)),
        ("p33x64_poisson", (33, 64), (1.0, 1.0), dict(poisson=0.25)),
        ("p17", (17,), (3.0,), {}),
    ]
    for name, nb, sizes, kw in periodic_cases:
        s = PeriodicFFTElasticHalfSpace(nb, 1.7, sizes, **kw)
        out[f"op_{name}_config"] = np.array(json.dumps(dict(
            kind="periodic", nb_grid_pts=list(nb), physical_sizes=list(sizes),
            young=1.7, kwargs=kw)))
        f = rng.standard_normal(nb)
        u = rng.standard_normal(nb)
        out[f"op_{name}_G"] = s.greens_function
        out[f"op_{name}_f"] = f
        out[f"op_{name}_u"] = u
        out[f"op_{name}_disp"] = s.evaluate_disp(f)
        out[f"op_{name}_force"] = s.evaluate_force(u)
    free_cases = [("f8x8", (8, 8), (1.0, 1.0)),
                  ("f7x9", (7, 9), (2.0, 1.0)),
                  ("f12x5", (12, 5), (1.0, 3.0))]
    for name, nb, sizes in free_cases:
        s = FreeFFTElasticHalfSpace(nb, 2.3, sizes)
        out[f"op_{name}_config"] = np.array(json.dumps(dict(
            kind="free", nb_grid_pts=list(nb), physical_sizes=list(sizes),
            young=2.3, kwargs={})))
        fpad = np.zeros(s.nb_domain_grid_pts)
        fpad[:nb[0], :nb[1]] = rng.standard_normal(nb)
        out[f"op_{name}_G"] = s.greens_function
        out[f"op_{name}_f"] = fpad
        out[f"op_{name}_disp"] = s.evaluate_disp(fpad)
        out[f"op_{name}_disp_unpadded"] = s.evaluate_disp(fpad[:nb[0], :nb[1]])
        upad = rng.standard_normal(s.nb_domain_grid_pts)
        out[f"op_{name}_u"] = upad
        out[f"op_{name}_force"] = s.evaluate_force(upad)

    # periodic grids with sides 3 * 2^m (the register-resident 3 * 2^m
    # passes), on their own random stream so the vectors above are unchanged
    rng3 = np.random.default_rng(20261204)
    for name, nb, sizes, kw in [("p96x96", (96, 96), (1.3, 0.7), {}),
                                ("p96x128_poisson", (96, 128), (2.0, 1.0), dict(poisson=0.3))]:
        s = PeriodicFFTElasticHalfSpace(nb, 1.7, sizes, **kw)
        out[f"op_{name}_config"] = np.array(json.dumps(dict(
            kind="periodic", nb_grid_pts=list(nb), physical_sizes=list(sizes),
            young=1.7, kwargs=kw)))
        f = rng3.standard_normal(nb)
        u = rng3.standard_normal(nb)
        out[f"op_{name}_G"] = s.greens_function
        out[f"op_{name}_f"] = f
        out[f"op_{name}_u"] = u
        out[f"op_{name}_disp"] = s.evaluate_disp(f)
        out[f"op_{name}_force"] = s.evaluate_force(u)

    # ---- solves -----------------------------------------------------------
    from refstubs import Topography, PlasticTopography

    def record(name, res, extra=None):
        out[f"ccg_{name}_x"] = res.x
        out[f"ccg_{name}_jac"] = res.jac
        out[f"ccg_{name}_active_set"] = res.active_set
        out[f"ccg_{name}_scalars"] = np.array(
            [res.offset, res.fun, res.nit, res.nfev, float(res.success)])
        if hasattr(res, "plastic"):
            out[f"ccg_{name}_plastic"] = res.plastic
        for k, v in (extra or {}).items():
            out[f"ccg_{name}_{k}"] = v

    def solve(name, substrate, heights, sizes, inputs, plastic_h=None, **kw):
        cfg = dict(kind="free" if isinstance(substrate, FreeFFTElasticHalfSpace)
                   else "periodic", nb_grid_pts=list(substrate.nb_grid_pts),
                   physical_sizes=list(sizes), young=substrate.young,
                   hardness=plastic_h, solver_kwargs=kw)
        out[f"ccg_{name}_config"] = np.array(json.dumps(cfg))
        topo = Topography(heights, sizes)
        if plastic_h is not None:
            topo = PlasticTopography(topo, plastic_h)
            system = PlasticNonSmoothContactSystem(substrate, topo)
        else:
            system = NonSmoothContactSystem(substrate, topo)
        res = system.minimize_proxy(**kw)
        extra = dict(heights=heights)
        if plastic_h is not None:
            extra["plastic_displ"] = topo.plastic_displ.copy()
        record(name, res, extra)
        out[f"ccg_{name}_inputs"] = np.array(inputs, dtype=float)

    # periodic Hertz, load control
    nb, sizes = (32, 32), (1.0, 1.0)
    h = _sphere(nb, sizes, 1.0)
    solve("hertz_periodic_load", PeriodicFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [np.nan, 1e-3, np.nan, 1e-12, 1e-14],
          external_force=1e-3, pentol=1e-12, forcetol=1e-14)
    # free sphere, offset control
    nb, sizes = (32, 28), (1.0, 1.0)
    h = _sphere(nb, sizes, 2.0)
    solve("sphere_free_offset", FreeFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [0.03, np.nan, np.nan, 1e-12, 1e-14],
          offset=0.03, pentol=1e-12, forcetol=1e-14)
    # a coarse free sphere that stalls: exercises the maxiter exit
    nb, sizes = (24, 20), (1.0, 1.0)
    h = _sphere(nb, sizes, 1.0)
    solve("stall_free_offset", FreeFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [0.01, np.nan, np.nan, 1e-9, 1e-14, 60],
          offset=0.01, pentol=1e-9, forcetol=1e-14, maxiter=60)
    # free sphere, load control
    nb, sizes = (16, 18), (2.0, 2.0)
    h = _sphere(nb, sizes, 2.0)
    solve("sphere_free_load", FreeFFTElasticHalfSpace(nb, 3.0, sizes),
          h, sizes, [np.nan, 0.05, np.nan, 1e-11, 1e-13],
          external_force=0.05, pentol=1e-11, forcetol=1e-13)
    # periodic rough, load control
    nb, sizes = (32, 32), (1.0, 1.0)
    h = self_affine(nb, sizes, 0.8, 0.1, seed=7)
    solve("rough_periodic_load", PeriodicFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [np.nan, 2e-3, np.nan, 1e-12, 1e-14],
          external_force=2e-3, pentol=1e-12, forcetol=1e-14)
    # periodic rough, plastic, load control (exercises the mixing branch)
    h = self_affine(nb, sizes, 0.7, 0.2, seed=11)
    solve("plastic_periodic_load", PeriodicFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [np.nan, 5e-3, 0.05, 1e-11, 1e-10], plastic_h=0.05,
          external_force=5e-3, pentol=1e-11, forcetol=1e-10, maxiter=2000)
    # periodic rough, plastic, offset control
    h = self_affine(nb, sizes, 0.7, 0.2, seed=12)
    off = float(np.max(h) - 0.3 * (np.max(h) - np.min(h)))
    solve("plastic_periodic_offset", PeriodicFFTElasticHalfSpace(nb, 1.0, sizes),
          h, sizes, [-off, np.nan, 0.05, 1e-11, 1e-10], plastic_h=0.05,
          offset=-off, pentol=1e-11, forcetol=1e-10, maxiter=2000)
    # Westergaard-like wavy profile, offset control
    nb, sizes = (64, 8), (30.0, 1.0)
    h = np.resize(np.cos(2 * np.pi * np.arange(nb[0]) / nb[0]), (nb[1], nb[0])).T.copy()
    solve("wavy_periodic_offset", PeriodicFFTElasticHalfSpace(nb, 3.56, sizes),
          h, sizes, [-0.5, np.nan, np.nan, 1e-9, 1e-5], offset=-0.5, pentol=1e-9)

    # ---- automated sweeps (PipelineFunction.contact_mechanics) -------------
    from ContactMechanics.PipelineFunction import contact_mechanics

    def pipeline(name, heights, sizes, periodic, hardness=None, **kw):
        cfg = dict(nb_grid_pts=list(heights.shape), physical_sizes=list(sizes),
                   periodic=periodic, hardness=hardness,
                   **{k: (list(v) if isinstance(v, (list, tuple, np.ndarray)) else v)
                      for k, v in kw.items()})
        out[f"pipe_{name}_config"] = np.array(json.dumps(cfg))
        out[f"pipe_{name}_heights"] = heights
        last = {}

        def cb(disp, gap, pressure, contacting, offset, load, area):
            last.update(disp=np.array(disp), gap=np.array(gap), pressure=np.array(pressure),
                        contacting=np.array(contacting),
                        scalars=np.array([offset, load, area], dtype=float))
        topo = Topography(heights, sizes, periodic=periodic)
        res = contact_mechanics(topo, hardness=hardness, results_callback=cb, **kw)
        for key, arr in zip(("mean_pressure", "area", "mean_displacement", "mean_gap",
                             "converged"), res):
            out[f"pipe_{name}_{key}"] = np.asarray(arr, dtype=float)
        for key, arr in last.items():
            out[f"pipe_{name}_last_{key}"] = arr

    nb, sizes = (32, 32), (1.0, 1.0)
    pipeline("pressures_periodic", self_affine(nb, sizes, 0.8, 0.1, seed=31), sizes, True,
             pressures=[2e-3, 1e-2], maxiter=2000, optimizer_kwargs=dict(forcetol=1e-13))
    nb, sizes = (24, 24), (1.0, 1.0)
    pipeline("nsteps_free", _sphere(nb, sizes, 2.0), sizes, False, nsteps=3, maxiter=2000,
             optimizer_kwargs=dict(forcetol=1e-13))
    nb, sizes = (32, 32), (1.0, 1.0)
    h = self_affine(nb, sizes, 0.7, 0.2, seed=32)
    span = float(np.max(h) - np.min(h))
    pipeline("offsets_plastic", h, sizes, True, hardness=0.05,
             offsets=[-(float(np.max(h)) - 0.2 * span), -(float(np.max(h)) - 0.35 * span)],
             maxiter=2000, optimizer_kwargs=dict(forcetol=1e-10))

    path = os.path.join(HERE, "reference_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


def main_semi(ref_root):
    """Golden vectors of SemiPeriodicFFTElasticHalfSpace (semi_vectors.npz)."""
    refstubs.install(ref_root)
    from ContactMechanics.FFTElasticHalfSpace import SemiPeriodicFFTElasticHalfSpace
    from ContactMechanics.Systems import NonSmoothContactSystem
    from refstubs import Topography

    rng = np.random.default_rng(20261204)
    out = {}
    cases = [
        ("s16x16_fp", (16, 16), (0.1, 0.1), (False, True), 10, 210e9),
        ("s12x9_pf", (12, 9), (1.0, 2.0), (True, False), 4, 1.0),
        ("s8x10_pp", (8, 10), (1.0, 1.0), (True, True), 3, 2.0),
        ("s9x8_ff", (9, 8), (1.0, 1.0), (False, False), 0, 1.0),
        ("s33x32_fp", (33, 32), (1.0, 1.0), (False, True), 10, 1.0),
    ]
    for name, nb, sizes, per, nim, young in cases:
        s = SemiPeriodicFFTElasticHalfSpace(nb, young, sizes, periodicity=per, n_images=nim)
        out[f"op_{name}_config"] = np.array(json.dumps(dict(
            kind="semi", nb_grid_pts=list(nb), physical_sizes=list(sizes), young=young,
            periodicity=list(per), n_images=nim, domain=list(s.nb_domain_grid_pts))))
        f = rng.standard_normal(nb)
        u = rng.standard_normal(s.nb_domain_grid_pts)
        out[f"op_{name}_G"] = s.greens_function
        out[f"op_{name}_f"] = f
        out[f"op_{name}_disp"] = s.evaluate_disp(f)
        out[f"op_{name}_disp_full"] = s.evaluate_disp(f, bIncludePadding=True)
        out[f"op_{name}_u"] = u
        out[f"op_{name}_force"] = s.evaluate_force(u)
        out[f"op_{name}_force_topo"] = s.evaluate_force(u[:nb[0], :nb[1]])
    # a load-controlled solve on a semi-periodic substrate: a cylinder-like
    # ridge (periodic along y, free along x)
    nb, sizes = (32, 24), (1.0, 1.0)
    x = ((np.arange(nb[0]) - nb[0] / 2) * sizes[0] / nb[0]).reshape(-1, 1)
    h = np.broadcast_to(-(x * x) / (2 * 1.5), nb).copy()
    h += 1e-3 * rng.standard_normal(nb)
    sub = SemiPeriodicFFTElasticHalfSpace(nb, 1.0, sizes, periodicity=(False, True), n_images=10)
    kw = dict(external_force=2e-3, pentol=1e-12, forcetol=1e-14)
    res = NonSmoothContactSystem(sub, Topography(h, sizes)).minimize_proxy(**kw)
    out["ccg_semi_ridge_config"] = np.array(json.dumps(dict(
        kind="semi", nb_grid_pts=list(nb), physical_sizes=list(sizes), young=1.0,
        periodicity=[False, True], n_images=10, solver_kwargs=kw)))
    out["ccg_semi_ridge_heights"] = h
    out["ccg_semi_ridge_x"] = res.x
    out["ccg_semi_ridge_jac"] = res.jac
    out["ccg_semi_ridge_active_set"] = res.active_set
    out["ccg_semi_ridge_scalars"] = np.array(
        [res.offset, res.fun, res.nit, res.nfev, float(res.success)])
    path = os.path.join(HERE, "semi_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


def main_kspace(ref_root):
    """Golden vectors of the k-space operators and energies (kspace_vectors.npz)."""
    refstubs.install(ref_root)
    from ContactMechanics import FreeFFTElasticHalfSpace, PeriodicFFTElasticHalfSpace

    rng = np.random.default_rng(20261205)
    out = {}
    cases = [("p16x12", PeriodicFFTElasticHalfSpace, (16, 12), (2.0, 1.5), dict(poisson=0.3)),
             ("p9x7", PeriodicFFTElasticHalfSpace, (9, 7), (1.0, 1.0), {}),
             ("p15", PeriodicFFTElasticHalfSpace, (15,), (2.0,), {}),
             ("f8x6", FreeFFTElasticHalfSpace, (8, 6), (1.0, 2.0), {})]
    for name, cls, nb, sizes, kw in cases:
        s = cls(nb, 1.3, sizes, **kw)
        dom = s.nb_domain_grid_pts
        out[f"k_{name}_config"] = np.array(json.dumps(dict(
            kind="free" if cls is FreeFFTElasticHalfSpace else "periodic",
            nb_grid_pts=list(nb), physical_sizes=list(sizes), young=1.3, kwargs=kw)))
        f = rng.standard_normal(dom)
        u = rng.standard_normal(dom)
        ka = s.evaluate_k_disp(f)
        kb = s.evaluate_k_force(u)
        out[f"k_{name}_f"] = f
        out[f"k_{name}_u"] = u
        out[f"k_{name}_kdisp"] = ka
        out[f"k_{name}_kforce"] = kb
        out[f"k_{name}_kforce_k"] = s.evaluate_k_force_k(ka)
        out[f"k_{name}_dot"] = np.array(s.evaluate_scalar_product_k_space(ka, kb))
        out[f"k_{name}_energy_k"] = np.array(s.evaluate(u, pot=True, forces=False)[0])
        e, fk = s.evaluate_k(ka, pot=True, forces=True)
        out[f"k_{name}_evaluate_k_energy"] = np.array(e)
    path = os.path.join(HERE, "kspace_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref = args[0] if args else os.environ.get("CM_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py /path/to/reference [--only=main|semi|kspace] "
                 "(or set CM_REFERENCE)")
    only = [a[7:] for a in sys.argv[1:] if a.startswith("--only=")]
    if not only or "main" in only:
        main(ref)
    if not only or "semi" in only:
        main_semi(ref)
    if not only or "kspace" in only:
        main_kspace(ref)
