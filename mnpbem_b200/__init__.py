"""mnpbem_b200 -- B200-native retarded BEM solve per wavelength.

Drop-in classes for the MNPBEM path ComParticle -> CompGreenRet ->
BEMRet(p).solve(exc.potential(p, enei)) -> exc.extinction / scattering.
"""
from .geometry import ComParticle, Particle, trisphere
from .materials import EpsConst, EpsDrude, EpsTable, EpsValues
from .planewave import CompStruct, PlaneWaveRet, SpectrumRet

__all__ = ["ComParticle", "Particle", "trisphere", "EpsConst", "EpsDrude", "EpsTable", "EpsValues",
           "CompStruct", "PlaneWaveRet", "SpectrumRet", "CompGreenRet", "BEMRet", "BEMRetIter"]


def __getattr__(name):
    # GPU-side classes are imported lazily so that geometry / materials work
    # without torch being imported.
    if name == "CompGreenRet":
        from .greenfun import CompGreenRet
        return CompGreenRet
    if name == "BEMRet":
        from .bem import BEMRet
        return BEMRet
    if name == "BEMRetIter":
        from .bem_iter import BEMRetIter
        return BEMRetIter
    raise AttributeError(name)
