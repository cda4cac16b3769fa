"""Automated contact sweeps (ContactMechanics/PipelineFunction.py:37-449).

``contact_mechanics`` steps a topography through a list of mean pressures,
a list of rigid-body offsets, or a number of automatically chosen offsets
(spaced so that the contact areas come out roughly evenly spaced on a log
scale), solving each step with the device solver, and returns the averaged
response.  Spatially resolved fields go to an optional callback.  Each step
is a fresh solve, as in the reference; with a hardness the plastic
displacement accumulates from step to step over listed loads or offsets and
is reset before every automatically chosen step.

The solver options travel in ``optimizer_kwargs`` (``precision="mixed"``
selects the mixed-precision solver).  The function is also available as the
method ``Topography.contact_mechanics``.
"""
import logging

import numpy as np

from .Factory import make_plastic_system, make_system
from .FFTElasticHalfSpace import FreeFFTElasticHalfSpace, PeriodicFFTElasticHalfSpace
from .Topography import PlasticTopography, Topography

_log = logging.getLogger(__name__)

MIN_PENTOL = 1e-12  # lower bound of the penetration tolerance (PipelineFunction.py:364)


def _numpy(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _contact_calculation(system, offset=None, external_force=None, history=None, pentol=None,
                         maxiter=None, optimizer_kwargs={}):
    """One solve at a given offset or load (PipelineFunction.py:37-135).

    Returns the displacement, gap, pressure and contact mask of the
    topography's grid, the offset, the mean pressure, the fractional contact
    area and the updated history (mean displacements, mean gaps, mean
    pressures, contact areas, convergence flags)."""
    topography = system.surface
    substrate = system.substrate
    middle = np.mean(topography.heights())
    if history is None:
        mean_displacements, mean_gaps, mean_pressures, total_contact_areas = [], [], [], []
        converged = np.array([], dtype=bool)
    else:
        mean_displacements, mean_gaps, mean_pressures, total_contact_areas, converged = history

    opt = system.minimize_proxy(offset=offset, external_force=external_force, pentol=pentol,
                                maxiter=maxiter, **optimizer_kwargs)
    force_xy = _numpy(opt.jac)
    displacement_xy = _numpy(opt.x)[:force_xy.shape[0], :force_xy.shape[1]]
    mean_displacements = np.append(mean_displacements, [opt.offset])
    mean_gaps = np.append(mean_gaps, [np.mean(displacement_xy) - middle - opt.offset])
    mean_load = force_xy.sum() / np.prod(topography.physical_sizes)
    mean_pressures = np.append(mean_pressures, [mean_load])
    total_contact_area = (force_xy > 0).sum() / np.prod(topography.nb_grid_pts)
    total_contact_areas = np.append(total_contact_areas, [total_contact_area])
    converged = np.append(converged, np.array([opt.success], dtype=bool))

    pressure_xy = force_xy / substrate.area_per_pt
    gap_xy = displacement_xy - topography.heights() - opt.offset
    gap_xy[gap_xy < 0.0] = 0.0
    contacting_points_xy = force_xy > 0
    return (displacement_xy, gap_xy, pressure_xy, contacting_points_xy, opt.offset, mean_load,
            total_contact_area,
            (mean_displacements, mean_gaps, mean_pressures, total_contact_areas, converged))


def _next_contact_step(system, history=None, pentol=None, maxiter=None, optimizer_kwargs={}):
    """A solve at an automatically chosen offset (PipelineFunction.py:138-226):
    first at minus the mean height, then just below the highest summit, then
    in the widest gap of the (log) contact areas found so far, or beyond the
    deepest offset when that gap is the last one."""
    topography = system.surface
    if hasattr(topography, "plastic_displ"):
        # steps are not in load order: every step starts from the elastic surface
        topography.plastic_displ = np.zeros_like(topography.plastic_displ)
    heights = topography.heights()
    top, middle, bot = np.max(heights), np.mean(heights), np.min(heights)
    step = 0 if history is None else len(history[0])
    if step == 0:
        mean_displacement = -middle
    elif step == 1:
        mean_displacement = -top + 0.01 * (top - middle)
    else:
        mean_displacements, _, _, total_contact_areas, _ = history
        sorted_disp, sorted_area = np.transpose(
            sorted(zip(mean_displacements, total_contact_areas), key=lambda pair: pair[1]))
        ref_area = np.log10(np.array(sorted_area + 1 / np.prod(topography.nb_grid_pts)))
        darea = np.append(ref_area[1:] - ref_area[:-1], -ref_area[-1])
        i = np.argmax(darea)
        if i == step - 1:
            mean_displacement = bot + 2 * (sorted_disp[-1] - bot)
        else:
            mean_displacement = (sorted_disp[i] + sorted_disp[i + 1]) / 2
    return _contact_calculation(system, offset=mean_displacement, pentol=pentol, maxiter=maxiter,
                                history=history, optimizer_kwargs=optimizer_kwargs)


def contact_mechanics(self, substrate=None, nsteps=None, offsets=None, pressures=None,
                      hardness=None, maxiter=100, results_callback=None, optimizer_kwargs={}):
    """Automated contact calculation on the topography ``self``
    (PipelineFunction.py:229-449).

    Exactly one of ``nsteps`` (automatically chosen offsets), ``offsets`` or
    ``pressures`` (mean pressures in units of E*) is given.  ``substrate`` is
    'periodic' or 'nonperiodic' (default from ``self.is_periodic``);
    ``hardness`` in units of E* makes the calculation plastic; ``maxiter``
    bounds each solve; ``results_callback(displacement_xy, gap_xy,
    pressure_xy, contacting_points_xy, mean_displacement, mean_pressure,
    total_contact_area)`` receives every step's fields.

    Returns mean pressure, total contact area, mean displacement, mean gap
    and convergence flags, one entry per step."""
    if substrate is None:
        substrate = "periodic" if self.is_periodic else "nonperiodic"
    if self.is_periodic != (substrate == "periodic"):
        if self.is_periodic:
            _log.warning("Topography is periodic, but the analysis is configured for free "
                         "boundaries.")
        else:
            _log.warning("Topography is not periodic, but the analysis is configured for "
                         "periodic boundaries.")
    given = [nsteps is not None, offsets is not None, pressures is not None]
    if not any(given):
        raise ValueError("Either `nsteps`, `offsets` or `pressures` must be given for a contact "
                         "mechanics calculation.")
    if all(given):
        raise ValueError("All of `nsteps`, `offsets` and `pressures` are given. There can only "
                         "be one.")
    if given[0] and given[1]:
        raise ValueError("Both of `nsteps` and `offsets` are given. Please specify only one.")
    if given[0] and given[2]:
        raise ValueError("Both of `nsteps` and `pressures` are given. Please specify only one.")
    if given[1] and given[2]:
        raise ValueError("Both of `offsets` and `pressures` are given. Please specify only one.")

    force_conv = np.prod(self.physical_sizes)
    plastic = hardness is not None and hardness > 0
    topography = PlasticTopography(self, hardness) if plastic else self
    half_space = dict(periodic=PeriodicFFTElasticHalfSpace, nonperiodic=FreeFFTElasticHalfSpace)
    half_space = half_space[substrate](topography.nb_grid_pts, 1.0, topography.physical_sizes)
    factory = make_plastic_system if plastic else make_system
    system = factory(substrate=half_space, surface=topography)

    # penetration tolerance from the roughness, whatever the units
    pentol = topography.rms_height_from_area() / (10 * np.mean(topography.nb_grid_pts))
    pentol = max(pentol, MIN_PENTOL)

    if pressures is not None:
        nsteps = len(pressures)
    if offsets is not None:
        nsteps = len(offsets)
    history = None
    for i in range(nsteps):
        if offsets is not None:
            step = _contact_calculation(system, offset=offsets[i], history=history, pentol=pentol,
                                        maxiter=maxiter, optimizer_kwargs=optimizer_kwargs)
        elif pressures is not None:
            step = _contact_calculation(system, external_force=pressures[i] * force_conv,
                                        history=history, pentol=pentol, maxiter=maxiter,
                                        optimizer_kwargs=optimizer_kwargs)
        else:
            step = _next_contact_step(system, history=history, pentol=pentol, maxiter=maxiter,
                                      optimizer_kwargs=optimizer_kwargs)
        history = step[-1]
        if results_callback is not None:
            results_callback(*step[:-1])

    mean_displacement, mean_gap, mean_pressure, total_contact_area, converged = history
    return (np.array(mean_pressure), np.array(total_contact_area), np.array(mean_displacement),
            np.array(mean_gap), np.array(converged))


# the reference registers the function on its topography interface
Topography.contact_mechanics = contact_mechanics
