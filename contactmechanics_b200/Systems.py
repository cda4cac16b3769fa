"""Contact systems (ContactMechanics/Systems.py, the non-smooth hard-wall path).

Besides the Polonsky-Keer solve behind ``minimize_proxy``, the system exposes
the reference's scipy-friendly objectives: the energy and forces of a
displacement field (``evaluate``, ``objective``), the primal objective with
the gap as variable and its Hessian product, and the dual objective with
the pressures as variable and its Hessian product (Systems.py:459-1008).
Their operator applications run on the device (the substrate's
``evaluate_force`` / ``evaluate_disp``); ``primal_minimize_proxy`` and
``dual_minimize_proxy`` drive scipy's L-BFGS-B with them.  The reference's
other two solvers for these objectives come from NuMPI
(``CCGWithoutRestart`` / ``CCGWithRestart``), which is not part of this
package.
"""
import numpy as np
import scipy.optimize as optim

from .FFTElasticHalfSpace import ElasticSubstrate
from .Optimization import constrained_conjugate_gradients


def _host(a):
    """A numpy view of a result field: torch tensors (CUDA or not) are copied
    to the host, numpy arrays pass through."""
    if hasattr(a, "detach") and hasattr(a, "cpu"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


class IncompatibleFormulationError(Exception):
    pass


class IncompatibleResolutionError(Exception):
    pass


class SystemBase(object):
    """Base class of contact systems (Systems.py:57-245)."""

    def __init__(self, substrate, surface):
        self.substrate = substrate
        self.area_per_pt = self.substrate.area_per_pt
        self.surface = surface
        self.dim = None
        self.gap = None
        self.disp = None
        self.comp_slice = self.substrate.local_topography_subdomain_slices

    _proxyclass = False

    @classmethod
    def is_proxy(cls):
        return cls._proxyclass

    @staticmethod
    def handles(substrate_type, surface_type, is_domain_decomposed):
        return False

    def compute_gap(self, disp, offset, *profile_args, **profile_kwargs):
        """Gap ``disp - (heights + offset)`` on the topography (Systems.py:123-134)."""
        return _host(disp)[self.comp_slice] - \
            (_host(self.surface.heights(*profile_args, **profile_kwargs)) + offset)

    def compute_contact_area(self):
        return self.compute_nb_contact_pts() * self.area_per_pt

    def compute_relative_contact_area(self):
        return self.compute_contact_area() / np.prod(self.substrate.physical_sizes)

    def shape_minimisation_input(self, in_array):
        """Flattened initial guess for scipy minimisers (Systems.py:162-180)."""
        if np.prod(self.substrate.nb_subdomain_grid_pts) == np.size(in_array):
            return np.ravel(_host(in_array))
        raise IncompatibleResolutionError()

    def shape_minimisation_output(self, in_array):
        """Minimiser output in the substrate's shape (Systems.py:182-196)."""
        if np.prod(self.substrate.nb_subdomain_grid_pts) == np.size(in_array):
            return np.reshape(_host(in_array), self.substrate.nb_subdomain_grid_pts)
        raise IncompatibleResolutionError()

    def _reshape_bounds(self, lbounds=None, ubounds=None):
        """scipy Bounds from (masked) bound arrays (Systems.py:198-210)."""
        if lbounds is not None and ubounds is not None:
            return optim.Bounds(lb=np.ma.filled(lbounds, -np.inf).ravel(),
                                ub=np.ma.filled(ubounds, np.inf).ravel())
        if lbounds is not None:
            return optim.Bounds(lb=np.ma.filled(lbounds, -np.inf).ravel())
        if ubounds is not None:
            return optim.Bounds(ub=np.ma.filled(ubounds, np.inf).ravel())
        return None

    def _lbounds_from_heights(self, offset):
        """Lower bounds of the displacements for gap >= 0 (Systems.py:212-222)."""
        lbounds = np.ma.masked_all(self.substrate.nb_subdomain_grid_pts)
        sl = self.substrate.local_topography_subdomain_slices
        lbounds.mask[sl] = False
        lbounds[sl] = _host(self.surface.heights()) + offset
        lbounds.set_fill_value(-np.inf)
        return lbounds


class NonSmoothContactSystem(SystemBase):
    """Hard-wall contact (Systems.py:370-611)."""

    def __init__(self, substrate, surface):
        super().__init__(substrate, surface)
        if tuple(surface.nb_grid_pts) != tuple(substrate.nb_grid_pts):
            raise IncompatibleResolutionError(
                "the substrate ({}) and the surface ({}) have incompatible nb_grid_ptss.".format(
                    substrate.nb_grid_pts, surface.nb_grid_pts))
        self.dim = len(self.substrate.nb_grid_pts)
        self.energy = None
        self.force = None
        self.contact_zone = None

    @staticmethod
    def handles(substrate_type, surface_type, is_domain_decomposed):
        return issubclass(substrate_type, ElasticSubstrate)

    @property
    def nb_grid_pts(self):
        return self.surface.nb_grid_pts

    def compute_normal_force(self):
        return float(np.sum(_host(self.substrate.force)))

    def compute_nb_contact_pts(self):
        return int(np.sum(_host(self.contact_zone)))

    def compute_contact_coordinates(self):
        return np.argwhere(_host(self.contact_zone))

    def logger_input(self):
        """Energy and total force for a Tools.Logger line (Systems.py:439-457)."""
        return (["energy", "force"], [self.energy, -float(np.sum(_host(self.substrate.force)))])

    def evaluate(self, disp, offset, pot=True, forces=False, logger=None):
        """Energy and/or forces of a displacement field (Systems.py:459-506)."""
        self.gap = self.compute_gap(disp, offset)
        self.substrate.compute(disp, pot, forces)
        self.energy = self.substrate.energy if pot else None
        self.force = self.substrate.force if forces else None
        if logger is not None:
            logger.st(*self.logger_input())
        return self.energy, self.force

    def objective(self, offset, disp0=None, gradient=False, logger=None):
        """A function of the displacements only, for scipy minimisers
        (Systems.py:508-549)."""
        res = self.substrate.nb_subdomain_grid_pts
        if gradient:
            def fun(disp):
                self.evaluate(np.reshape(disp, res), offset, forces=True, logger=logger)
                return self.energy, -np.ravel(_host(self.force))
        else:
            def fun(disp):
                return self.evaluate(np.reshape(disp, res), offset, forces=False, logger=logger)[0]
        return fun

    def hessian_product(self, disp):
        return self.primal_hessian_product(disp)

    def primal_objective(self, offset, gradient=True):
        """Energy (and minus the forces) as a function of the gap
        (Systems.py:613-660)."""
        res = self.substrate.nb_subdomain_grid_pts
        heights = _host(self.surface.heights())
        if gradient:
            def fun(gap):
                disp = np.reshape(gap, res) + heights + offset
                self.evaluate(disp, offset, forces=True)
                return self.energy, -np.ravel(_host(self.force))
        else:
            def fun(gap):
                disp = np.reshape(gap, res) + heights + offset
                return self.evaluate(disp, offset, forces=False)[0]
        return fun

    def primal_hessian_product(self, gap):
        """Hessian of the primal objective applied to a gap field: minus the
        forces of that field (Systems.py:662-686)."""
        shape = np.shape(gap)
        res = self.substrate.nb_subdomain_grid_pts
        return np.reshape(-_host(self.substrate.evaluate_force(np.reshape(gap, res))), shape)

    def primal_minimize_proxy(self, offset, init_gap=None, solver="l-bfgs-b", gtol=1e-8,
                              maxiter=1000):
        """Minimise the primal objective with the gap as variable
        (Systems.py:688-757); solver 'l-bfgs-b'."""
        self._check_solver(solver)
        self.disp = self.force = self.contact_zone = None
        self.init_gap = init_gap
        bnds = self._reshape_bounds(np.zeros(np.shape(init_gap)))
        result = optim.minimize(self.primal_objective(offset, gradient=True),
                                self.shape_minimisation_input(init_gap), method="L-BFGS-B",
                                jac=True, bounds=bnds,
                                options=dict(gtol=gtol, ftol=1e-20, maxiter=maxiter))
        if result.success:
            self.offset = offset
            self.gap = result.x
            self.force = self.substrate.force = result.jac
            self.contact_zone = result.x == 0
            self.disp = self.gap + offset + np.reshape(_host(self.surface.heights()),
                                                       self.gap.shape)
        return result

    def evaluate_dual(self, force, offset, logger=None):
        """Energy and gap of a pressure field (Systems.py:759-830)."""
        disp = _host(self.substrate.evaluate_disp(-force))
        heights = _host(self.surface.heights())
        self.gradient = disp - heights - offset
        self.energy = 0.5 * np.sum(force * disp) - np.sum(force * (heights + offset))
        self.substrate.force = -force
        self.substrate.disp = disp
        if logger is not None:
            n = np.prod(self.nb_grid_pts)
            f = -self.substrate.force[self.substrate.local_topography_subdomain_slices]
            proj = self.gradient * (force > 0)
            logger.st(["energy", "force", "frac_rep_area", "frac_att_area", "max_residual",
                       "rms_residual"],
                      [self.energy, -np.sum(self.substrate.force), np.sum(f > 0) / n,
                       np.sum(f < 0) / n, np.max(np.abs(proj)),
                       np.sqrt(np.sum(proj ** 2) / n)])
        return self.energy, self.gradient

    def dual_objective(self, offset, gradient=True, logger=None):
        """Energy and gap as a function of the pressures (Systems.py:832-882)."""
        res = self.substrate.topography_nb_subdomain_grid_pts
        if not gradient:
            raise NotImplementedError

        def fun(pressure):
            self.evaluate_dual(np.reshape(pressure, res), offset, logger=logger)
            return self.energy, np.ravel(self.gradient)
        return fun

    def dual_hessian_product(self, pressure):
        """Hessian of the dual objective applied to a pressure field: its
        displacements (Systems.py:884-904)."""
        shape = np.shape(pressure)
        res = self.substrate.topography_nb_subdomain_grid_pts
        return np.reshape(_host(self.substrate.evaluate_disp(-np.reshape(pressure, res))), shape)

    def dual_minimize_proxy(self, offset, init_force=None, solver="l-bfgs-b", gtol=1e-8,
                            maxiter=1000, logger=None):
        """Minimise the dual objective with the pixel forces as variables
        (Systems.py:906-978); solver 'l-bfgs-b'."""
        self._check_solver(solver)
        self.disp = self.force = self.contact_zone = None
        self.init_force = init_force
        if init_force is not None and \
                np.shape(init_force) != tuple(self.substrate.topography_nb_subdomain_grid_pts):
            raise IncompatibleResolutionError
        bnds = self._reshape_bounds(np.zeros(np.shape(init_force)))
        result = optim.minimize(self.dual_objective(offset, gradient=True, logger=logger),
                                np.ravel(init_force), method="L-BFGS-B", jac=True, bounds=bnds,
                                options=dict(gtol=gtol, ftol=1e-20, maxiter=maxiter))
        if result.success:
            self.offset = offset
            self.gap = result.jac
            self.force = self.substrate.force = result.x
            self.contact_zone = result.x > 0
            self.disp = self.gap + offset + np.reshape(_host(self.surface.heights()),
                                                       self.gap.shape)
        return result

    @staticmethod
    def _check_solver(solver):
        solvers = {"ccg-without-restart", "ccg-with-restart", "l-bfgs-b"}
        if solver not in solvers:
            raise ValueError("Input correct solver name from {}".format(solvers))
        if solver != "l-bfgs-b":
            raise NotImplementedError(
                "solver '{}' comes from NuMPI, which this package does not include; use "
                "'l-bfgs-b', or minimize_proxy for the Polonsky-Keer solve".format(solver))

    def minimize_proxy(self, solver=constrained_conjugate_gradients, **kwargs):
        """Run ``solver(substrate, surface, **kwargs)`` and store the solution
        (Systems.py:572-611)."""
        self.disp = None
        self.force = None
        self.contact_zone = None
        result = solver(self.substrate, self.surface, **kwargs)
        if result.success:
            self.offset = result.offset
            self.disp = result.x
            self.force = self.substrate.force = result.jac
            self.contact_zone = result.jac > 0
            self.substrate.check()
        return result
