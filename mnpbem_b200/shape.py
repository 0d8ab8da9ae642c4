"""Derivatives of the extinction cross section with respect to the mesh vertices.

The geometry of a face is fixed by its nodes: ``verts2`` (corners, edge
midpoints and quad centres) for curved particles, ``verts`` for flat ones.
The vertex array of a compound particle is those arrays of its particles,
stacked.  For a direction D in that space (one (nvert, 3) displacement) the
directional derivative of ext follows from the BEM system A(v) x = b(v) and
the far-field functional z(x, v), ext = 4 pi / k Im(pol* . z):

    dx = A^-1 (db - dA x),     dz = z(dx, v) + dz/dv|_x D.

The solve reuses the factors already built for the wavelength (one more solve
per direction, no new factorisation).  dA x, db and the explicit far-field
term come from the GPU assembly recomputed at v +- h D: every Green, derivative
and refinement tile is rebuilt on the fly by the assembly kernels, none is
stored per direction, and dA x is formed as (A(v+hD) x - A(v-hD) x) / 2h by the
FP64 operator kernel (bem200_bem_apply), which is second-order accurate in h.
The refinement pattern (which face pairs get the near-field integrals) is
piecewise constant in v; it is taken at v, and a step that would change it
raises an error.

``ExtinctionShape`` wraps this as a torch.autograd.Function of the
coefficients t of a displacement v + sum_k t_k D_k: forward gives ext, the
backward pass the gradient over the K directions (K extra solves), and jvp the
forward-mode product.  The reference has no gradients; the derivative is checked
against central finite differences of the whole solver along seeded random
directions (tests/test_shape_gpu.py).
"""
import copy
import ctypes

import numpy as np

from . import _native as nat
from .greenfun import CompGreenRet

_CACHES = ("_b200_face_cache", "_b200_side_cache")


def _curved(q):
    return q.interp == "curv" and q.verts2 is not None


def vertex_array(cp):
    """The (nvert, 3) node coordinates that fix the geometry of ``cp``: verts2
    of its curved particles, verts of its flat ones, stacked in particle order."""
    return np.vstack([(q.verts2 if _curved(q) else q.verts) for q in cp.p])


def perturbed(cp, delta):
    """Copy of the compound particle with its vertex array moved by ``delta``.
    Corner vertices of curved particles (used only to classify near pairs)
    stay where they are."""
    delta = np.asarray(delta, dtype=float).reshape(-1, 3)
    if len(delta) != len(vertex_array(cp)):
        raise ValueError("perturbed: delta has {} rows, the vertex array {}".format(len(delta),
                                                                                     len(vertex_array(cp))))
    new = copy.copy(cp)
    parts, off = [], 0
    for q in cp.p:
        r = copy.copy(q)
        for a in _CACHES:
            r.__dict__.pop(a, None)
        if _curved(q):
            m = len(q.verts2)
            r.verts2 = q.verts2 + delta[off:off + m]
        else:
            m = len(q.verts)
            r.verts = q.verts + delta[off:off + m]
        off += m
        r._norm()
        parts.append(r)
    new.p = parts
    for a in _CACHES:
        new.__dict__.pop(a, None)
    new._build()
    return new


def random_directions(cp, k, seed=0):
    """k seeded random unit directions in the vertex space of ``cp``, (k, nvert, 3)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((k,) + vertex_array(cp).shape)
    return d / np.sqrt(np.sum(d * d, axis=(1, 2), keepdims=True))


def _farfield_z(exc, p, enei, W1, W2):
    from .adjoint import _pe
    return _pe(exc, p, enei, W1, W2)


class _Operator:
    """A(M, e, n) x of the BEM system for a fixed x (bem200_bem_apply)."""

    def __init__(self, bem, npol, W1, W2):
        import torch
        self.bem, self.npol = bem, npol
        self.x = torch.cat([W1.reshape(-1), W2.reshape(-1)])
        n = bem.n
        self.scr = torch.empty(int(nat.lib().bem200_bem_apply_workspace_size(n, npol)), dtype=torch.uint8,
                               device=bem.dev)

    def __call__(self, mats, nvec):
        import torch
        bem = self.bem
        n, npol = bem.n, self.npol
        out = torch.empty(8 * n * npol, dtype=torch.complex128, device=bem.dev)
        xb = self.x.data_ptr()
        nat.call("bem200_bem_apply", n, npol, *[nat.ptr(m) for m in mats], bem._eps_mode, bem._e1p, bem._e2p,
                 nat.ptr(nvec), bem.k, ctypes.c_void_p(xb), ctypes.c_void_p(xb + 16 * 4 * n * npol), None,
                 nat.ptr(out), nat.ptr(self.scr), nat.stream_ptr())
        return out


class ShapeSensitivity:
    """Directional derivatives of the extinction of ``bem.p`` along fixed
    vertex directions, for any number of wavelengths.

    Construction builds, once per direction and sign, the moved particle
    v +- h D and its Green function (refinement tables on the GPU; they do not
    depend on the wavelength).  ``extinction(exc, enei)`` then costs, per
    direction, two matrix assemblies, two FP64 operator products and one solve
    with the wavelength's factors."""

    def __init__(self, bem, directions, h=1e-4):
        import torch
        p = bem.p
        D = np.asarray(directions, dtype=float)
        D = D[None] if D.ndim == 2 else D
        if D.shape[1:] != vertex_array(p).shape:
            raise ValueError("ShapeSensitivity: directions must be (K, {}, 3)".format(len(vertex_array(p))))
        self.bem, self.D, self.h = bem, D, float(h)
        base = bem.g.refined
        self.sides = []
        for d in D:
            pair = []
            for sign in (1.0, -1.0):
                cp = perturbed(p, sign * self.h * d)
                g = CompGreenRet(cp, cp, **bem.options)
                r = g.refined
                if r.nref != base.nref or not (torch.equal(r.row[:r.nref], base.row[:r.nref]) and
                                               torch.equal(r.col[:r.nref], base.col[:r.nref])):
                    raise RuntimeError("ShapeSensitivity: the step changes the near-pair pattern; use a smaller h")
                nvec = torch.as_tensor(np.ascontiguousarray(cp.nvec), dtype=torch.float64, device=bem.dev)
                pair.append((cp, g, nvec))
            self.sides.append(pair)

    def extinction(self, exc, enei):
        """ext (npol,) and dext (K, npol) at wavelength ``enei``."""
        bem, h = self.bem, self.h
        p = bem.p
        bem.init(enei)
        bt, npol = exc.rhs_device(p, enei, bem._eps_mode, bem._e1p, bem._e2p, device=bem.dev)
        W1, W2 = bem.solve_device(bt, npol)
        z, km = _farfield_z(exc, p, enei, W1, W2)
        ext = np.real(4 * np.pi / km * np.imag(z))
        op = _Operator(bem, npol, W1, W2)
        dext = np.zeros((len(self.D), npol))
        for k, pair in enumerate(self.sides):
            parts = []
            for cp, g, nvec in pair:
                mats = g.bem_matrices(bem.enei, dtype="c128")
                Ax = op(mats, nvec)
                del mats
                b, _ = exc.rhs_device(cp, enei, bem._eps_mode, bem._e1p, bem._e2p, device=bem.dev)
                zz, _ = _farfield_z(exc, cp, enei, W1, W2)
                parts.append((Ax, b, zz))
            (Ap, bp, zp), (Am, bm, zm) = parts
            rhs = ((bp - bm) - (Ap - Am)) / (2 * h)
            dW1, dW2 = bem.solve_device(rhs, npol)
            dz, _ = _farfield_z(exc, p, enei, dW1, dW2)
            dz = dz + (zp - zm) / (2 * h)
            dext[k] = np.real(4 * np.pi / km * np.imag(dz))
        return ext, dext


def extinction_shape_derivative(bem, exc, enei, directions, h=1e-4):
    """Extinction at ``enei`` and its directional derivatives along
    ``directions`` ((K, nvert, 3) or (nvert, 3), in the vertex space of
    bem.p; nm per unit coefficient).  ``bem`` is a BEMRet (fp64 or mixed),
    ``h`` the assembly step in nm.  Returns (ext (npol,), dext (K, npol))."""
    return ShapeSensitivity(bem, directions, h).extinction(exc, enei)


class ExtinctionShape:
    """torch.autograd.Function: ext = ExtinctionShape.apply(t, bem, exc, enei, directions)

    ext (npol,) of the particle with vertices v + sum_k t_k D_k, t a float64
    tensor of K coefficients.  At t = 0 the wavelength's solver ``bem`` is used
    as it is; otherwise a solver of the same precision is built for the moved
    particle.  backward returns d ext / d t (K directional derivatives, each one
    more solve with the factors); jvp returns sum_k tangent_k d ext / d t_k."""

    @staticmethod
    def apply(t, bem, exc, enei, directions, h=1e-4):
        import torch
        D = np.asarray(directions, dtype=float)
        D = D[None] if D.ndim == 2 else D

        def solver_at(tv):
            if not np.any(tv):
                return bem
            from .bem import BEMRet
            moved = perturbed(bem.p, np.tensordot(tv, D, axes=1))
            return BEMRet(moved, precision=bem.precision, engine=bem.engine, ir_tol=bem.ir_tol,
                          ir_maxit=bem.ir_maxit, **bem.options)

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, tt):
                tv = tt.detach().cpu().numpy().astype(float)
                if tv.shape != (len(D),):
                    raise ValueError("ExtinctionShape: t must have one entry per direction")
                ext, dext = extinction_shape_derivative(solver_at(tv), exc, enei, D, h)
                jac = torch.as_tensor(dext, dtype=torch.float64)    # (K, npol)
                ctx.save_for_backward(jac)
                ctx.jac = jac
                return torch.as_tensor(ext, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gout):
                (jac,) = ctx.saved_tensors
                return (jac @ gout.to(jac.dtype).cpu().reshape(-1)).to(gout.device)

            @staticmethod
            def jvp(ctx, tangent):
                jac = ctx.jac
                return tangent.to(jac.dtype).cpu().reshape(-1) @ jac

        return _F.apply(t)
