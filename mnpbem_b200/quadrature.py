"""Quadrature rules for boundary-element integration.

Two families are needed by the retarded Green-function refinement:

* a 28-point rule of polynomial degree 11 on the unit triangle
  {(x, y): x, y >= 0, x + y <= 1}, used to integrate over neighbouring faces
  (reference: mnpbem/utils/quadrature.py:92-198, rule 18; MATLAB
  Misc/integration/@quadface/private/triangle_unit_set.m);
* a polar (radial x angular) rule built from Legendre-Gauss-Lobatto nodes,
  centred on the face centroid, used for the weakly singular self term
  (reference: mnpbem/utils/quadface.py:106-249).

Weights follow the reference convention: the triangle rule sums to 1, the
polar triangle rule sums to 1 and the polar quadrilateral rule sums to 4
(the area of [-1, 1]^2).
"""
import numpy as np


def lgl_nodes(n):
    """Legendre-Gauss-Lobatto nodes and weights on [-1, 1] (n + 1 points).

    Newton iteration on x P_n(x) - P_{n-1}(x) = 0 started from the
    Chebyshev-Gauss-Lobatto points (reference: mnpbem/utils/quadrature.py:15-89).
    """
    if n < 2:
        raise ValueError("lgl_nodes: need n >= 2")
    n1 = n + 1
    x = np.cos(np.pi * np.arange(n1) / n)
    p = np.zeros((n1, n1))
    xold = 2.0 * np.ones(n1)
    while np.max(np.abs(x - xold)) > np.finfo(float).eps:
        xold = x.copy()
        p[:, 0] = 1.0
        p[:, 1] = x
        for k in range(2, n1):
            p[:, k] = ((2 * k - 1) * x * p[:, k - 1] - (k - 1) * p[:, k - 2]) / k
        x = xold - (x * p[:, n] - p[:, n - 1]) / (n1 * p[:, n])
    w = 2.0 / (n * n1 * p[:, n] ** 2)
    return x, w


def triangle_rule28():
    """28-point, degree-11 rule on the unit triangle; weights sum to 1.

    The node/weight table is the published rule that MNPBEM selects as its
    default (``rule=18``); the numbers must be identical for the Green-function
    refinement to agree with the reference (mnpbem/utils/quadrature.py:159-198).
    Orbits: centroid, 3 edge-type orbits of size 3 (a, b, b), and one orbit of
    size 6 repeated over three parameter sets.
    """
    third = 1.0 / 3.0
    # size-3 orbits: (p, q, q) and permutations
    orbit3 = [
        (0.9480217181434233, 0.02598914092828833, 0.008744311553736190),
        (0.8114249947041546, 0.09428750264792270, 0.03808157199393533),
        (0.01072644996557060, 0.4946367750172147, 0.01885544805613125),
        (0.5853132347709715, 0.2073433826145142, 0.07215969754474100),
        (0.1221843885990187, 0.4389078057004907, 0.06932913870553720),
    ]
    # size-6 orbits: all (a, b) placements with c = 1 - a - b
    orbit6 = [
        (0.6779376548825902, 0.04484167758913055, 0.27722066752827925, 0.04105631542928860),
        (0.8588702812826364, 0.0, 0.1411297187173636, 0.007362383783300573),
    ]
    xs, ys, ws = [third], [third], [0.08797730116222190]
    for p_, q_, w_ in orbit3:
        xs += [p_, q_, q_]
        ys += [q_, p_, q_]
        ws += [w_, w_, w_]
    for a, b, c, w_ in orbit6:
        # placements in the order x = [a a b b c c], y = [b c a c a b]
        xs += [a, a, b, b, c, c]
        ys += [b, c, a, c, a, b]
        ws += [w_] * 6
    x = np.array(xs)
    y = np.array(ys)
    w = np.array(ws)
    return x, y, w / np.sum(w)


def polar_triangle(npol=(7, 5)):
    """Polar rule on the unit triangle around its centroid (3 sectors of 60 deg).

    Radial LGL nodes on (0, 1], angular LGL nodes on a 60 degree sector, three
    copies rotated by 120 degrees, mapped to unit-triangle coordinates.
    Weights include the polar Jacobian and are normalised to sum 1
    (reference: mnpbem/utils/quadface.py:106-182).
    """
    n_rad, n_ang = _npol_pair(npol)
    x1, w1 = lgl_nodes(n_rad)
    rho = 0.5 * (x1 + 1 + 1e-6)
    x2, w2 = lgl_nodes(n_ang)
    phi = np.deg2rad(270 + 60 * x2)
    phi0 = np.deg2rad(120)
    rho_g, phi_g = np.meshgrid(rho, phi, indexing="ij")
    rho_f = rho_g.ravel()
    phi_f = phi_g.ravel()
    rad = 1.0 / np.abs(2 * np.sin(phi_f))
    ph = np.hstack([phi_f, phi_f + phi0, phi_f + 2 * phi0])
    rho3 = np.tile(rho_f, 3)
    rad3 = np.tile(rad, 3)
    xp = np.cos(ph) * rho3 * rad3
    yp = np.sin(ph) * rho3 * rad3
    x = (1 - np.sqrt(3) * xp - yp) / 3
    y = (1 + np.sqrt(3) * xp - yp) / 3
    w = np.tile(np.outer(w1, w2).ravel() * rho_f * rad ** 2, 3)
    return x, y, w / np.sum(w)


def polar_quad(npol=(7, 5)):
    """Polar rule on [-1, 1]^2 around the centre (4 sectors of 90 deg).

    Weights are normalised to sum 4 (reference: mnpbem/utils/quadface.py:184-249).
    """
    n_rad, n_ang = _npol_pair(npol)
    x1, w1 = lgl_nodes(n_rad)
    rho = 0.5 * (x1 + 1 + 1e-6)
    x2, w2 = lgl_nodes(n_ang)
    phi = np.deg2rad(90 + 45 * x2)
    phi0 = np.deg2rad(90)
    rho_g, phi_g = np.meshgrid(rho, phi, indexing="ij")
    rho_f = rho_g.ravel()
    phi_f = phi_g.ravel()
    rad = 1.0 / np.abs(np.sin(phi_f))
    ph = np.hstack([phi_f, phi_f + phi0, phi_f + 2 * phi0, phi_f + 3 * phi0])
    rho4 = np.tile(rho_f, 4)
    rad4 = np.tile(rad, 4)
    x = np.cos(ph) * rho4 * rad4
    y = np.sin(ph) * rho4 * rad4
    w = np.tile(np.outer(w1, w2).ravel() * rho_f * rad ** 2, 4)
    return x, y, 4 * w / np.sum(w)


def _npol_pair(npol):
    if np.isscalar(npol):
        return int(npol), int(npol)
    return int(npol[0]), int(npol[1])


class QuadFace:
    """Integration rules attached to a particle (reference: mnpbem/utils/quadface.py:47-103).

    x, y, w   : 28-point triangle rule (sum w = 1)
    x3, y3, w3: polar rule on triangles (sum w3 = 1)
    x4, y4, w4: polar rule on quadrilaterals (sum w4 = 4)
    """

    def __init__(self, rule=18, npol=(7, 5), refine=None):
        if rule != 18:
            raise NotImplementedError("QuadFace: only the default 28-point rule (rule=18) is supported")
        if refine is not None and refine > 1:
            raise NotImplementedError("QuadFace: 'refine' subdivision is not supported")
        self.npol = _npol_pair(npol)
        self.x, self.y, self.w = triangle_rule28()
        self.x3, self.y3, self.w3 = polar_triangle(self.npol)
        self.x4, self.y4, self.w4 = polar_quad(self.npol)
