"""System factories (ContactMechanics/Factory.py:42-156)."""
from .FFTElasticHalfSpace import FreeFFTElasticHalfSpace, PeriodicFFTElasticHalfSpace
from .PlasticSystemSpecialisations import PlasticNonSmoothContactSystem
from .Systems import NonSmoothContactSystem


def _make_system_args(surface, substrate=None, communicator=None, physical_sizes=None,
                      fft="mpi", **kwargs):
    if isinstance(surface, str) or hasattr(surface, "read"):
        raise NotImplementedError("reading topography files is not part of this package")
    nb_grid_pts = surface.nb_grid_pts
    if physical_sizes is None:
        physical_sizes = getattr(surface, "physical_sizes", None)
        if physical_sizes is None:
            raise ValueError("physical sizes neither provided in input or in file")
    if substrate is None:
        substrate = "periodic" if surface.is_periodic else "free"
    if substrate == "periodic":
        substrate = PeriodicFFTElasticHalfSpace(nb_grid_pts, physical_sizes=physical_sizes,
                                                communicator=communicator, **kwargs)
    elif substrate == "free":
        substrate = FreeFFTElasticHalfSpace(nb_grid_pts, physical_sizes=physical_sizes,
                                            communicator=communicator, **kwargs)
    return substrate, surface


def make_system(*args, **kwargs):
    substrate, surface = _make_system_args(*args, **kwargs)
    return NonSmoothContactSystem(substrate=substrate, surface=surface)


def make_plastic_system(*args, **kwargs):
    substrate, surface = _make_system_args(*args, **kwargs)
    return PlasticNonSmoothContactSystem(substrate=substrate, surface=surface)
