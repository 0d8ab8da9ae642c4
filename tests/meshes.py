"""Seeded test meshes shared by the CPU and GPU tests."""
import contextlib

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


# Reference mesh-generator cases pinned by tests/golden/meshes.npz:
# tag -> (generator, args, kwargs)
MESH_CASES = {
    "ell": ("triellipsoid", (400, [10.0, 15.0, 25.0]), {}),
    "seg": ("trispheresegment", (np.linspace(0, np.pi, 7), np.linspace(0, np.pi / 2, 5), 10.0),
            {"triangles": True, "interp": "curv"}),
    "rod": ("trirod", (20.0, 60.0, [13, 6, 9]), {"interp": "curv"}),
    "rodtri": ("trirod", (12.0, 30.0, [9, 5, 5]), {"triangles": True, "interp": "curv"}),
    "cube": ("tricube", (6, 40.0, 0.25), {"interp": "curv"}),
    "rod2400": ("trirod", (20.0, 80.0, [41, 16, 31]), {"interp": "curv"}),
    "cube25k": ("tricube", (66, 100.0, 0.25), {"interp": "curv"}),
}


def shape_particle(tag, eps_b=1.77, drude=DRUDE_AU):
    """ComParticle of one reference-generator case in a medium eps_b.
    'rodbem' = trirod(12, 30, [9, 5, 5]) and 'cubebem' = tricube(5, 20, 0.25),
    both curved, and 'ellbem' = triellipsoid(60, [4, 6, 9]), flat, are the
    meshes whose BEM results the fixtures hold."""
    from mnpbem_b200 import geometry
    extra = {"rodbem": ("trirod", (12.0, 30.0, [9, 5, 5]), {"interp": "curv"}),
             "cubebem": ("tricube", (5, 20.0, 0.25), {"interp": "curv"}),
             "ellbem": ("triellipsoid", (60, [4.0, 6.0, 9.0]), {})}
    name, args, kw = extra[tag] if tag in extra else MESH_CASES[tag]
    part = getattr(geometry, name)(*args, **kw)
    return ComParticle([EpsConst(eps_b), EpsDrude(*drude)], [part], [[2, 1]], 1, interp=kw.get("interp", "flat"))


def face_nodes(p):
    """Per-face node coordinates (n, 9, 3), NaN where a face has no such node."""
    f, v = (p.faces, p.verts) if p.faces2 is None else (p.faces2, p.verts2)
    out = np.full((len(f), 9, 3), np.nan)
    ok = ~np.isnan(f)
    out[:, :f.shape[1]][ok] = v[f[ok].astype(int)]
    return out


@contextlib.contextmanager
def refinement_of(base):
    """Meshes solved inside this context refine exactly the face pairs that
    `base` refines (the selection of bem200_refine_count / _fill is made from
    base's centroids and boundary radii).  The reverse-mode gradient holds the
    refinement pattern fixed, so central differences of perturbed meshes must
    too: on fine meshes some pair distances cross the cutoff within a step of
    1e-3 nm, and the quadrature switch of such a pair is a jump in ext."""
    import torch
    from mnpbem_b200 import _native as nat
    f64 = dict(dtype=torch.float64, device="cuda")
    pos0 = torch.as_tensor(np.ascontiguousarray(base.pos), **f64)
    rad0 = torch.as_tensor(np.ascontiguousarray(base.bradius()), **f64)
    real = nat.call

    def call(name, *args):
        if name in ("bem200_refine_count", "bem200_refine_fill"):
            args = (args[0], nat.ptr(pos0), nat.ptr(rad0)) + tuple(args[3:])
        return real(name, *args)
    nat.call = call
    try:
        yield
    finally:
        nat.call = real
