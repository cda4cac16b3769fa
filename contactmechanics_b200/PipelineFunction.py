"""Automated contact sweeps (the ``contact_mechanics`` pipeline function of
ContactMechanics/PipelineFunction.py:229-449).

A sweep steps one topography through a list of mean pressures, a list of
rigid-body offsets, or a number of automatically placed offsets, solving
each step with the device solver, and reports per step the mean pressure,
the fractional contact area, the offset (mean displacement), the mean gap
and whether the solve converged.

Organisation:

* :class:`StepRecord` is one step's outcome; a sweep keeps them in a list in
  the order the steps were solved and turns the list into the five returned
  arrays at the end.
* :func:`next_offset` is a pure function of the records so far and of the
  topography's height statistics: it places the automatic steps, first at
  minus the mean height, then just below the highest summit, then into the
  widest gap of the log contact areas found so far (or beyond the deepest
  offset when the widest gap is the one above the largest area) -- the
  placement rule of PipelineFunction.py:138-226, which the reference's
  recorded sweeps pin down.
* :class:`_Sweep` owns the contact system and the solver settings and turns
  one solve into a record (:meth:`_Sweep.solve`); the spatially resolved
  fields of a step are only assembled when a ``results_callback`` wants them.

Each step is a fresh solve, as in the reference.  With a hardness the
plastic displacement accumulates from step to step over listed loads or
offsets and is cleared before every automatically placed step (those steps
are not in load order).  Solver options travel in ``optimizer_kwargs``
(``precision="mixed"`` selects the mixed-precision solver).  The function is
also available as the method ``Topography.contact_mechanics``.
"""
import logging
from typing import NamedTuple

import numpy as np

from .Factory import make_plastic_system, make_system
from .FFTElasticHalfSpace import FreeFFTElasticHalfSpace, PeriodicFFTElasticHalfSpace
from .Systems import _host
from .Topography import PlasticTopography, Topography

_log = logging.getLogger(__name__)

# smallest penetration tolerance a sweep hands to the solver
# (PipelineFunction.py:364)
MIN_PENTOL = 1e-12

_SUBSTRATES = {"periodic": PeriodicFFTElasticHalfSpace, "nonperiodic": FreeFFTElasticHalfSpace}


class StepRecord(NamedTuple):
    """Outcome of one step of a sweep."""
    offset: float          # rigid-body offset (the reported mean displacement)
    mean_gap: float        # mean displacement - mean height - offset
    mean_pressure: float   # total force / nominal area
    area: float            # fraction of the grid points in contact
    converged: bool


class HeightStats(NamedTuple):
    top: float
    mean: float
    bottom: float
    points: int


def height_stats(heights):
    h = _host(heights)
    return HeightStats(float(h.max()), float(h.mean()), float(h.min()), int(h.size))


def next_offset(records, stats):
    """Offset of the next automatically placed step given the steps solved so
    far (any order) and the topography's height statistics."""
    n = len(records)
    if n == 0:
        return -stats.mean
    if n == 1:
        return -stats.top + 0.01 * (stats.top - stats.mean)
    offsets = np.array([r.offset for r in records])
    areas = np.array([r.area for r in records])
    order = np.argsort(areas, kind="stable")  # ties keep the order of solving
    offsets, areas = offsets[order], areas[order]
    log_area = np.log10(areas + 1.0 / stats.points)
    # spacing between neighbouring areas, and beyond the largest one the
    # distance to full contact (log10 1 = 0)
    spacing = np.concatenate([np.diff(log_area), [-log_area[-1]]])
    widest = int(np.argmax(spacing))
    if widest == n - 1:
        # push beyond the deepest offset, doubling its distance to the bottom
        return stats.bottom + 2.0 * (offsets[-1] - stats.bottom)
    return 0.5 * (offsets[widest] + offsets[widest + 1])


class _Sweep:
    """The system of a sweep and the settings every one of its solves uses."""

    def __init__(self, system, pentol, maxiter, optimizer_kwargs, results_callback):
        self.system = system
        self.pentol = pentol
        self.maxiter = maxiter
        self.optimizer_kwargs = dict(optimizer_kwargs or {})
        self.results_callback = results_callback
        self.records = []

    @property
    def topography(self):
        return self.system.surface

    def solve(self, offset=None, external_force=None):
        """Solve one step, record it and hand its fields to the callback."""
        topo = self.topography
        mean_height = float(np.mean(_host(topo.heights())))
        res = self.system.minimize_proxy(offset=offset, external_force=external_force,
                                         pentol=self.pentol, maxiter=self.maxiter,
                                         **self.optimizer_kwargs)
        force = _host(res.jac)
        # displacements on the topography's part of the domain
        disp = _host(res.x)[tuple(slice(0, n) for n in force.shape)]
        nominal_area = float(np.prod(topo.physical_sizes))
        rec = StepRecord(offset=float(res.offset),
                         mean_gap=float(disp.mean()) - mean_height - float(res.offset),
                         mean_pressure=float(force.sum()) / nominal_area,
                         area=float(np.count_nonzero(force > 0)) / force.size,
                         converged=bool(res.success))
        self.records.append(rec)
        if self.results_callback is not None:
            gap = disp - _host(topo.heights()) - rec.offset
            np.maximum(gap, 0.0, out=gap)
            self.results_callback(disp, gap, force / self.system.substrate.area_per_pt,
                                  force > 0, rec.offset, rec.mean_pressure, rec.area)
        return rec

    def solve_auto(self):
        """Solve at the next automatically placed offset; the plastic
        displacement starts from zero."""
        topo = self.topography
        if hasattr(topo, "plastic_displ"):
            topo.plastic_displ = np.zeros_like(topo.plastic_displ)
        return self.solve(offset=next_offset(self.records, height_stats(topo.heights())))

    def arrays(self):
        """(mean pressure, contact area, mean displacement, mean gap, converged)."""
        r = self.records
        return (np.array([x.mean_pressure for x in r]), np.array([x.area for x in r]),
                np.array([x.offset for x in r]), np.array([x.mean_gap for x in r]),
                np.array([x.converged for x in r], dtype=bool))


def _check_step_arguments(nsteps, offsets, pressures):
    given = [name for name, v in (("nsteps", nsteps), ("offsets", offsets),
                                  ("pressures", pressures)) if v is not None]
    if not given:
        raise ValueError("Either `nsteps`, `offsets` or `pressures` must be given for a contact "
                         "mechanics calculation.")
    if len(given) == 3:
        raise ValueError("All of `nsteps`, `offsets` and `pressures` are given. There can only "
                         "be one.")
    if len(given) == 2:
        raise ValueError("Both of `{}` and `{}` are given. Please specify only one."
                         .format(*given))


def contact_mechanics(self, substrate=None, nsteps=None, offsets=None, pressures=None,
                      hardness=None, maxiter=100, results_callback=None, optimizer_kwargs={}):
    """Automated contact calculation on the topography ``self``
    (PipelineFunction.py:229-449).

    Exactly one of ``nsteps`` (automatically placed offsets), ``offsets`` or
    ``pressures`` (mean pressures in units of E*) is given.  ``substrate`` is
    'periodic' or 'nonperiodic' (default from ``self.is_periodic``);
    ``hardness`` in units of E* makes the calculation plastic; ``maxiter``
    bounds each solve; ``results_callback(displacement_xy, gap_xy,
    pressure_xy, contacting_points_xy, mean_displacement, mean_pressure,
    total_contact_area)`` receives every step's fields.

    Returns mean pressure, total contact area, mean displacement, mean gap
    and convergence flags, one entry per step in the order solved."""
    if substrate is None:
        substrate = "periodic" if self.is_periodic else "nonperiodic"
    if self.is_periodic != (substrate == "periodic"):
        _log.warning("Topography is {}periodic, but the analysis is configured for {} "
                     "boundaries.".format("" if self.is_periodic else "not ",
                                          "free" if self.is_periodic else "periodic"))
    _check_step_arguments(nsteps, offsets, pressures)

    plastic = hardness is not None and hardness > 0
    topography = PlasticTopography(self, hardness) if plastic else self
    half_space = _SUBSTRATES[substrate](topography.nb_grid_pts, 1.0, topography.physical_sizes)
    system = (make_plastic_system if plastic else make_system)(substrate=half_space,
                                                               surface=topography)
    # penetration tolerance from the roughness, whatever the height units
    pentol = max(topography.rms_height_from_area() / (10 * np.mean(topography.nb_grid_pts)),
                 MIN_PENTOL)
    sweep = _Sweep(system, pentol, maxiter, optimizer_kwargs, results_callback)
    if pressures is not None:
        force_per_pressure = float(np.prod(self.physical_sizes))
        for p in pressures:
            sweep.solve(external_force=p * force_per_pressure)
    elif offsets is not None:
        for off in offsets:
            sweep.solve(offset=off)
    else:
        for _ in range(nsteps):
            sweep.solve_auto()
    return sweep.arrays()


# the reference registers the function on its topography interface
Topography.contact_mechanics = contact_mechanics
