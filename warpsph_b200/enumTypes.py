"""Scheme enumerations, same names and values as the reference's src/warpSPH/enumTypes.py:1-66."""
from enum import Enum


class EnergyScheme(Enum):
    equalWork = 0
    PdV = 1
    diminishing = 2
    monotonic = 3
    hybrid = 4
    CRK = 5


class AdaptiveSupportScheme(Enum):
    NoScheme = 0
    Monaghan = 1
    Owen = 2


class ViscositySwitch(Enum):
    Balsara1995 = 0
    Colagrossi2004 = 1
    CullenDehnen2010 = 2
    CullenHopkins = 3
    MorrisMonaghan1997 = 4
    Rosswog2000 = 5
    NoneSwitch = 6


class CompressibleSPHScheme(Enum):
    Monaghan = 0
    CompSPH = 1
    CRKSPH = 2


class WeaklyCompressibleSPHScheme(Enum):
    deltaSPH = 0


class IncompressibleSPHScheme(Enum):
    divergenceFree = 0


class EquationOfState(Enum):
    stiffTait = "stiffTait"
    Tait = "Tait"
    isoThermal = "isoThermal"
    Polytropic = "polytropic"
    Murnaghan = "murnaghan"


class DensityDiffusionScheme(Enum):
    deltaSPH = 0
    denormalized = 1
    densityOnly = 2
    deltaOnly = 3
    denormalizedOnly = 4


class PressureForceScheme(Enum):
    conservative = 0
    nonConservative = 1
    Antuono = 2
    i = 3
    j = 4
    symmetric = 5
