"""Optimization algorithms (ContactMechanics/Optimization/__init__.py)."""
from .ConstrainedConjugateGradients import (constrained_conjugate_gradients,  # noqa: F401
                                            constrained_conjugate_gradients_batch)
