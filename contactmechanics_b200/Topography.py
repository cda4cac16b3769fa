"""Minimal topography containers for the contact path.

The reference takes its surfaces from SurfaceTopography (``Topography``,
``PlasticTopography``), which is not part of this package.  These classes
provide the attributes the contact path reads: ``heights()``,
``nb_grid_pts``, ``physical_sizes``, ``area_per_pt``, ``is_periodic``,
``rms_height_from_area()``; the plastic container adds ``hardness``,
``plastic_displ`` and ``plastic_area`` (the plastic system accumulates the
negative plastic gap into ``plastic_displ``,
PlasticSystemSpecialisations.py:68, so ``heights()`` returns the original
heights plus ``plastic_displ``).
"""
import numpy as np


class Topography:
    def __init__(self, heights, physical_sizes, periodic=True, **kwargs):
        self._heights = np.asarray(heights, dtype=np.float64)
        if not hasattr(physical_sizes, "__iter__"):
            physical_sizes = (physical_sizes,)
        self.physical_sizes = tuple(float(s) for s in physical_sizes)
        self.is_periodic = bool(periodic)

    @property
    def nb_grid_pts(self):
        return self._heights.shape

    @property
    def nb_subdomain_grid_pts(self):
        return self._heights.shape

    @property
    def subdomain_locations(self):
        return (0,) * self._heights.ndim

    @property
    def subdomain_slices(self):
        return tuple(slice(0, n) for n in self.nb_grid_pts)

    @property
    def dim(self):
        return self._heights.ndim

    @property
    def area_per_pt(self):
        return np.prod(self.physical_sizes) / np.prod(self.nb_grid_pts)

    def heights(self):
        return self._heights

    def rms_height_from_area(self):
        h = self._heights
        return float(np.sqrt(np.mean((h - h.mean()) ** 2)))


class PlasticTopography(Topography):
    def __init__(self, topography, hardness, plastic_displ=None):
        super().__init__(topography.heights(), topography.physical_sizes,
                         periodic=topography.is_periodic)
        self.parent_topography = topography
        self.hardness = hardness
        self.plastic_displ = (np.zeros(self.nb_grid_pts) if plastic_displ is None
                              else np.asarray(plastic_displ, dtype=np.float64))

    def heights(self):
        return self._heights + self.plastic_displ

    @property
    def plastic_area(self):
        return np.count_nonzero(self.plastic_displ) * self.area_per_pt
