"""Substrate base classes (names and behaviour of ContactMechanics/Substrates.py)."""
import abc


class Substrate(object, metaclass=abc.ABCMeta):
    """Generic base class of all substrates (Substrates.py:34-111)."""
    _periodic = None

    class Error(Exception):
        pass

    name = "generic_halfspace"

    def spawn_child(self, dummy):
        raise self.Error("Only substrates with free boundaries can do this")

    @classmethod
    def is_periodic(cls):
        if cls._periodic is not None:
            return cls._periodic
        raise cls.Error(
            "periodicity of Substrate type '{}' ('{}') is not defined".format(cls.name, cls.__name__))

    @property
    @abc.abstractmethod
    def nb_domain_grid_pts(self):
        pass

    @property
    @abc.abstractmethod
    def nb_subdomain_grid_pts(self):
        pass

    @property
    @abc.abstractmethod
    def subdomain_locations(self):
        pass

    @property
    @abc.abstractmethod
    def communicator(self):
        pass

    def check(self, force=None):
        """All forces are acceptable for a generic substrate (Substrates.py:93-111)."""


class ElasticSubstrate(Substrate, metaclass=abc.ABCMeta):
    """Elastic substrate: stores energy and forces (Substrates.py:114-177)."""
    name = "generic_elastic_halfspace"

    def __init__(self):
        self.energy = None
        self.force = None
        self.force_k = None

    def compute(self, disp, pot=True, forces=False):
        self.energy, self.force = self.evaluate(disp, pot, forces)

    def compute_k(self, disp_k, pot=True, forces=False):
        """Energy and/or forces from a displacement field in Fourier space
        (Substrates.py:151-166)."""
        self.energy, self.force_k = self.evaluate_k(disp_k, pot, forces)

    def evaluate_k(self, disp_k, pot=True, forces=False):
        raise NotImplementedError()

    def evaluate(self, disp, pot=True, forces=False):
        raise NotImplementedError()


class PlasticSubstrate(Substrate):
    """Plastic substrate marker class (Substrates.py:180-184)."""
    name = "generic_plastic_halfspace"
