"""Seeded test meshes shared by the CPU and GPU tests."""
import numpy as np

from mnpbem_b200.geometry import ComParticle, trisphere
from mnpbem_b200.materials import EpsConst, EpsDrude

DRUDE_AU = (9.84, 9.0, 0.067)


def sphere(n=144, diameter=20.0, eps_b=1.0):
    """Config-0 geometry: trisphere(n, d), Drude gold in a medium eps_b."""
    return ComParticle([EpsConst(eps_b), EpsDrude(*DRUDE_AU)], [trisphere(n, diameter)], [[2, 1]], 1,
                       interp="curv")


def dimer(n=144, diameter=10.0, gap=2.0, eps_b=1.77):
    """Two spheres on the x axis with a surface gap `gap` (config-1 family)."""
    a, b = trisphere(n, diameter), trisphere(n, diameter)
    a.shift([-(diameter / 2 + gap / 2), 0, 0])
    b.shift([diameter / 2 + gap / 2, 0, 0])
    return ComParticle([EpsConst(eps_b), EpsDrude(*DRUDE_AU)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
