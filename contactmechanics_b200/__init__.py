"""B200-native elastic contact solve with the ContactMechanics API.

The FFT Green's-function half-spaces and the Polonsky-Keer constrained
conjugate-gradient solver of ContactEngineering/ContactMechanics, running
as hand-written sm_100a CUDA in ``lib/libcm_b200.so`` behind the
reference's Substrates / Systems / Optimization call signatures.
"""
from .Substrates import ElasticSubstrate, PlasticSubstrate, Substrate  # noqa: F401
from .FFTElasticHalfSpace import (FreeFFTElasticHalfSpace,  # noqa: F401
                                  PeriodicFFTElasticHalfSpace,
                                  SemiPeriodicFFTElasticHalfSpace)
from .Optimization import (constrained_conjugate_gradients,  # noqa: F401
                           constrained_conjugate_gradients_batch)
from .Systems import NonSmoothContactSystem  # noqa: F401
from .PlasticSystemSpecialisations import PlasticNonSmoothContactSystem  # noqa: F401
from .Factory import make_plastic_system, make_system  # noqa: F401
from .Topography import PlasticTopography, Topography  # noqa: F401
from .PipelineFunction import contact_mechanics  # noqa: F401

__version__ = "0.1.0"
