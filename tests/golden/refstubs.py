"""Serial stand-ins for the reference's absent third-party modules.

Test infrastructure only.  ContactMechanics (the reference) imports muGrid,
NuMPI, SurfaceTopography and DiscoverVersion; none is installed in this
image.  ``install(reference_root)`` registers minimal serial replacements in
``sys.modules`` and puts the unmodified reference package on ``sys.path`` so
that ``make_golden.py`` can run the reference's own hot-path code to produce
golden vectors.  Each stand-in follows the contract the reference's call
sites need:

* ``muGrid.FFTEngine`` -- ``fft`` is ``numpy.fft.rfftn(a, axes=(1, 0))``
  (unnormalised, half spectrum along axis 0; ContactMechanics/
  FFTElasticHalfSpace.py:104-128, pinned by test/test_fft_elastic_half_space.py
  :356-371), ``ifft`` the unnormalised inverse, ``normalisation = 1/N``.
* ``NuMPI.Tools.Reduction`` -- serial sum/max/min/all/dot.
* ``SurfaceTopography`` -- ``Topography`` / ``PlasticTopography`` holding a
  height array; ``PlasticTopography.heights()`` adds ``plastic_displ`` (the
  reference accumulates the negative plastic gap into it,
  PlasticSystemSpecialisations.py:68).
"""
import sys
import types

import numpy as np


def _module(name):
    mod = types.ModuleType(name)
    sys.modules[name] = mod
    return mod


class _Field:
    def __init__(self, shape, dtype):
        self.p = np.zeros(shape, dtype=dtype)


class FFTEngine:
    def __init__(self, nb_grid_pts, comm=None):
        self.nb_domain_grid_pts = tuple(int(n) for n in nb_grid_pts)
        self.nb_subdomain_grid_pts = self.nb_domain_grid_pts
        self.subdomain_locations = (0,) * len(self.nb_domain_grid_pts)
        four = list(self.nb_domain_grid_pts)
        four[0] = four[0] // 2 + 1
        self._cpp = types.SimpleNamespace(
            nb_fourier_subdomain_grid_pts=tuple(four),
            fourier_subdomain_locations=(0,) * len(four))
        self.normalisation = 1.0 / float(np.prod(self.nb_domain_grid_pts))
        self._axes = tuple(reversed(range(len(self.nb_domain_grid_pts))))

    def real_space_field(self, name):
        return _Field(self.nb_domain_grid_pts, float)

    def fourier_space_field(self, name):
        return _Field(self._cpp.nb_fourier_subdomain_grid_pts, complex)

    def fft(self, real, fourier):
        fourier.p[...] = np.fft.rfftn(real.p, axes=self._axes)

    def ifft(self, fourier, real):
        s = [self.nb_domain_grid_pts[a] for a in self._axes]
        real.p[...] = np.fft.irfftn(fourier.p, s=s, axes=self._axes) \
            * np.prod(self.nb_domain_grid_pts)


class Reduction:
    def __init__(self, comm=None):
        self.comm = comm

    def sum(self, a, *args, **kw):
        return np.sum(a, *args, **kw)

    def max(self, a, *args, **kw):
        return np.max(a, *args, **kw)

    def min(self, a, *args, **kw):
        return np.min(a, *args, **kw)

    def all(self, a):
        return np.all(a)

    def any(self, a):
        return np.any(a)

    def dot(self, a, b):
        return np.dot(a, b)


class _Comm:
    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    rank = 0
    size = 1


class Topography:
    is_periodic = True

    def __init__(self, heights, physical_sizes, periodic=True, **kw):
        self._heights = np.asarray(heights, dtype=float)
        if not hasattr(physical_sizes, "__iter__"):
            physical_sizes = (physical_sizes,)
        self.physical_sizes = tuple(float(s) for s in physical_sizes)
        self.is_periodic = periodic
        self.nb_grid_pts = self._heights.shape
        self.nb_subdomain_grid_pts = self._heights.shape
        self.subdomain_locations = (0,) * self._heights.ndim
        self.subdomain_slices = tuple(slice(0, n) for n in self.nb_grid_pts)

    def heights(self):
        return self._heights

    @property
    def area_per_pt(self):
        return np.prod(self.physical_sizes) / np.prod(self.nb_grid_pts)

    def rms_height_from_area(self):
        h = self._heights
        return np.sqrt(np.mean((h - h.mean()) ** 2))


class PlasticTopography(Topography):
    def __init__(self, topography, hardness, plastic_displ=None):
        super().__init__(topography.heights(), topography.physical_sizes,
                         periodic=topography.is_periodic)
        self.parent = topography
        self.hardness = hardness
        self.plastic_displ = (np.zeros(self.nb_grid_pts) if plastic_displ is None
                              else plastic_displ)

    def heights(self):
        return self._heights + self.plastic_displ

    @property
    def plastic_area(self):
        return np.count_nonzero(self.plastic_displ) * self.area_per_pt


def install(reference_root):
    """Register the stand-ins and make the reference importable."""
    if "muGrid" not in sys.modules:
        mg = _module("muGrid")
        mg.FFTEngine = FFTEngine
        mg.Communicator = lambda comm=None: comm

        numpi = _module("NuMPI")
        mpi = types.SimpleNamespace(COMM_WORLD=_Comm(), COMM_SELF=_Comm())
        numpi.MPI = mpi
        tools = _module("NuMPI.Tools")
        tools.Reduction = Reduction
        red = _module("NuMPI.Tools.Reduction")
        red.Reduction = Reduction
        numpi.Tools = tools
        opt = _module("NuMPI.Optimization")
        opt.CCGWithoutRestart = None
        opt.CCGWithRestart = None
        numpi.Optimization = opt

        st = _module("SurfaceTopography")
        st.Topography = Topography
        st.PlasticTopography = PlasticTopography
        st.UniformLineScan = None
        st.open_topography = None

        class UniformTopographyInterface:
            @staticmethod
            def register_function(name, fn):
                pass

        st.UniformTopographyInterface = UniformTopographyInterface
        hc = _module("SurfaceTopography.HeightContainer")
        hc.UniformTopographyInterface = UniformTopographyInterface
        st.HeightContainer = hc
        sup = _module("SurfaceTopography.Support")

        def doi(*args):
            def deco(f):
                return f
            return deco

        sup.doi = doi
        st.Support = sup
        io = _module("SurfaceTopography.IO")
        io.ReaderBase = type("ReaderBase", (), {})
        st.IO = io

        dv = _module("DiscoverVersion")
        dv.get_version = lambda *a, **k: "0+stub"
    if reference_root not in sys.path:
        sys.path.insert(0, reference_root)
