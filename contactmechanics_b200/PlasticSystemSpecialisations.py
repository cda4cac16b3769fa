"""Plastic hard-wall contact (ContactMechanics/PlasticSystemSpecialisations.py)."""
import numpy as np

from .FFTElasticHalfSpace import ElasticSubstrate
from .Systems import NonSmoothContactSystem, _host
from .Topography import PlasticTopography


class PlasticNonSmoothContactSystem(NonSmoothContactSystem):
    """Penetration-hardness model (PlasticSystemSpecialisations.py:37-69)."""

    @staticmethod
    def handles(substrate_type, surface_type, is_domain_decomposed):
        return issubclass(substrate_type, ElasticSubstrate) and \
            issubclass(surface_type, PlasticTopography)

    def minimize_proxy(self, **kwargs):
        # the solver works with forces: convert the hardness (a pressure)
        hardness = self.surface.hardness * self.surface.area_per_pt
        opt = super().minimize_proxy(hardness=hardness, **kwargs)
        if opt.success:
            self.surface.plastic_displ += np.where(
                _host(opt.plastic), self.compute_gap(self.disp, self.offset), 0.)
        return opt
