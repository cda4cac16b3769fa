"""Contact systems (ContactMechanics/Systems.py, the non-smooth hard-wall path)."""
import numpy as np

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
