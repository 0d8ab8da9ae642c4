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


# ---------------------------------------------------------------------------
# Reverse mode: the gradient over every vertex coordinate from one transposed
# solve.  With A(v) x = b(v) and z = w(v)^T x (bilinear pairings),
#     dz/dv = w_v^T x + lambda^T (b_v - A_v x),     lambda = A^-T w,
# where lambda^T A_v x is contracted on the GPU over all face pairs at once
# (bem200_shape_gradient: far pairs analytically, refined pairs through the
# exact derivatives of their quadrature), and the geometry chain
# v -> (centroids, normals, tangents, areas, face nodes) and the plane-wave
# terms w_v, b_v run as torch autograd on the device.

def _torch_norm(v):
    import torch
    return torch.clamp_min(torch.linalg.vector_norm(v, dim=-1, keepdim=True), 1e-14)


def face_geometry(cp, V):
    """Differentiable face data of ``cp`` from its vertex array V (torch,
    (nvert, 3), the layout of ``vertex_array``): pos, nvec, tvec1, tvec2
    (n, 3), area (n,) and the node table (n, 9, 3) of the refinement kernels.
    The same formulas as the particle's own _norm_curv / _norm_flat and
    quad_integration (reference particle.py:464-614, :1431-1575)."""
    import torch
    from .geometry import tri6_deriv
    dev, f64 = V.device, V.dtype
    outs = {k: [] for k in ("pos", "nvec", "tvec1", "tvec2", "area", "nodes")}
    off = 0
    for q in cp.p:
        nf = q.nfaces
        ind3, ind4 = q.index34()
        if _curved(q):
            m = len(q.verts2)
            Vq = V[off:off + m]
            f2 = q.faces2
            tri = np.zeros((nf, 6), dtype=np.int64)
            tri[ind3] = f2[ind3][:, [0, 1, 2, 4, 5, 6]].astype(np.int64)
            tri[ind4] = f2[ind4][:, [0, 1, 2, 4, 5, 8]].astype(np.int64)
            vb = Vq[torch.as_tensor(tri, device=dev)]                      # (nf, 6, 3)
            c = torch.tensor([-1, -1, -1, 4, 4, 4], dtype=f64, device=dev) / 9
            cx = torch.tensor([1, 0, -1, 4, -4, 0], dtype=f64, device=dev) / 3
            cy = torch.tensor([0, 1, -1, 4, 0, -4], dtype=f64, device=dev) / 3
            cx4 = torch.tensor([1, 0, -1, 0, 0, 0], dtype=f64, device=dev)
            cy4 = torch.tensor([0, -1, -1, 2, 2, -2], dtype=f64, device=dev)
            is4 = torch.zeros(nf, dtype=torch.bool, device=dev)
            is4[torch.as_tensor(ind4, device=dev)] = True
            pos = torch.where(is4[:, None], vb[:, 5], torch.einsum("c,icd->id", c, vb))
            v1 = torch.where(is4[:, None], torch.einsum("c,icd->id", cy4, vb), torch.einsum("c,icd->id", cy, vb))
            v2 = torch.where(is4[:, None], torch.einsum("c,icd->id", cx4, vb), torch.einsum("c,icd->id", cx, vb))
            nv = torch.linalg.cross(v1, v2)
            nv = nv / _torch_norm(nv)
            v1 = v1 / _torch_norm(v1)
            v2 = torch.linalg.cross(nv, v1)
            # area: 28-point rule on the curved sub-triangles (quads: two of them)
            qr = q.quad
            dx, dy = tri6_deriv(qr.x, qr.y)
            dxt, dyt = torch.as_tensor(dx, device=dev), torch.as_tensor(dy, device=dev)
            wq = torch.as_tensor(qr.w, device=dev)

            def sub_area(vbs):
                px = torch.einsum("tc,icd->itd", dxt, vbs)
                py = torch.einsum("tc,icd->itd", dyt, vbs)
                jac = torch.linalg.vector_norm(torch.linalg.cross(px, py, dim=2), dim=2)
                return (0.5 * wq[None, :] * jac).sum(dim=1)
            area = sub_area(vb)
            if len(ind4):
                t2 = f2[ind4][:, [2, 3, 0, 6, 7, 8]].astype(np.int64)
                extra = torch.zeros(nf, dtype=f64, device=dev)
                extra = extra.index_add(0, torch.as_tensor(ind4, device=dev), sub_area(Vq[torch.as_tensor(t2, device=dev)]))
                area = area + extra
            ntab = np.zeros((nf, 9), dtype=np.int64)
            ntab[ind3, :6] = f2[ind3][:, [0, 1, 2, 4, 5, 6]].astype(np.int64)
            ntab[ind4, :9] = f2[ind4][:, :9].astype(np.int64)
            valid = np.zeros((nf, 9), dtype=bool)
            valid[ind3, :6] = True
            valid[ind4, :9] = True
        else:
            m = len(q.verts)
            Vq = V[off:off + m]
            fa = q.faces
            c3 = fa[:, :3].astype(np.int64)
            corners = Vq[torch.as_tensor(c3, device=dev)]
            is4 = torch.zeros(nf, dtype=torch.bool, device=dev)
            is4[torch.as_tensor(ind4, device=dev)] = True
            c4 = np.where(np.isnan(fa[:, 3]), 0, fa[:, 3]).astype(np.int64)
            v4 = Vq[torch.as_tensor(c4, device=dev)]
            pos = torch.where(is4[:, None], (corners.sum(dim=1) + v4) / 4.0, corners.sum(dim=1) / 3.0)

            def frame(a, b, cc):
                e1, e2 = a - b, cc - b
                nn = torch.linalg.cross(e1, e2)
                ar = 0.5 * torch.linalg.vector_norm(nn, dim=1)
                nn = nn / _torch_norm(nn)
                e1 = e1 / _torch_norm(e1)
                return ar, e1, torch.linalg.cross(nn, e1), nn
            a1, t1a, t2a, na = frame(corners[:, 0], corners[:, 1], corners[:, 2])
            a2, t1b, t2b, nb = frame(corners[:, 2], v4, corners[:, 0])
            a2 = torch.where(is4, a2, torch.zeros_like(a2))
            area = a1 + a2
            big = (is4 & (a2 > a1))[:, None]
            v1, v2, nv = torch.where(big, t1b, t1a), torch.where(big, t2b, t2a), torch.where(big, nb, na)
            ntab = np.zeros((nf, 9), dtype=np.int64)
            ntab[:, :3] = c3
            ntab[ind4, 3] = fa[ind4, 3].astype(np.int64)
            valid = np.zeros((nf, 9), dtype=bool)
            valid[:, :3] = True
            valid[ind4, 3] = True
        nodes = Vq[torch.as_tensor(ntab, device=dev)] * torch.as_tensor(valid, device=dev)[:, :, None]
        for k, val in (("pos", pos), ("nvec", nv), ("tvec1", v1), ("tvec2", v2), ("area", area), ("nodes", nodes)):
            outs[k].append(val)
        off += m
    return {k: torch.cat(v) for k, v in outs.items()}


def _planewave_terms(cp, exc, enei, pos, nvec, area):
    """Right-hand side b (the layout of BEMRet.rhs, complex (8 n p)) and the
    extinction weights w (solution layout [W1 | W2], (8 n p)) of the plane
    wave as torch functions of the face data (reference
    planewave_ret.py:257-361, bem_ret.py:1360-1429, spectrum_ret.py:231-392)."""
    import torch
    dev = pos.device
    n = cp.n
    pol = torch.as_tensor(np.asarray(exc.pol, dtype=complex), device=dev)
    dirs = torch.as_tensor(np.asarray(exc.dir, dtype=float), device=dev)
    npol = pol.shape[0]
    k0 = 2 * np.pi / enei
    eps_m = complex(np.asarray(cp.eps[exc.medium - 1](enei)[0]).ravel()[0])
    km = k0 * np.sqrt(eps_m)
    io = np.asarray(cp.inout_faces)
    e1 = torch.as_tensor(np.asarray(cp.eps1(enei), dtype=complex), device=dev)[:, None]
    e2 = torch.as_tensor(np.asarray(cp.eps2(enei), dtype=complex), device=dev)[:, None]
    posc = pos.to(torch.complex128)
    ph = torch.exp(1j * km * (posc @ dirs.T.to(torch.complex128))) / (1j * k0)          # (n, p)
    ndir = nvec.to(torch.complex128) @ dirs.T.to(torch.complex128)                        # (n, p)
    a_side, ap_side = [], []
    for side in range(2):
        on = torch.as_tensor((io[:, side] == exc.medium).astype(float), device=dev)[:, None]
        a = (ph * on)[:, None, :] * pol.T[None, :, :]                                     # (n, 3, p)
        ap = (1j * km * ndir)[:, None, :] * a
        a_side.append(a)
        ap_side.append(ap)
    a = a_side[1] - a_side[0]
    alpha = ap_side[1] - ap_side[0]
    nvc = nvec.to(torch.complex128)
    De = -1j * k0 * (torch.einsum("ic,icp->ip", nvc, a_side[1]) * e2 - torch.einsum("ic,icp->ip", nvc, a_side[0]) * e1)
    b = torch.cat([torch.zeros(n * npol, dtype=torch.complex128, device=dev), a.reshape(-1), alpha.reshape(-1),
                   De.reshape(-1)])
    # far-field weights of z_q = conj(pol_q) . e_far(dir_q)
    phase = torch.exp(-1j * km * (posc @ dirs.T.to(torch.complex128))) * area.to(torch.complex128)[:, None]
    pc = torch.conj(pol)
    pcd = (pc * dirs.to(torch.complex128)).sum(dim=1)                                     # (p,)
    Ws = []
    for side in range(2):
        on = torch.as_tensor((io[:, side] == exc.medium).astype(float), device=dev)[:, None]
        ws = -1j * km * pcd[None, :] * phase * on                                         # (n, p)
        wh = 1j * k0 * (phase * on)[:, None, :] * pc.T[None, :, :]                        # (n, 3, p)
        Ws.append(torch.cat([ws, wh.reshape(n, 3 * npol)], dim=1))                        # (n, 4p)
    w = torch.cat([Ws[0].reshape(-1), Ws[1].reshape(-1)])
    return b, w, km


def _transposed_solve(bem, w, npol, tol=1e-12, maxit=30):
    """lambda = A^-T w for the current wavelength's factors: one transposed
    solve with the complex128 factors (fp64), or refinement of the complex64
    transposed solve against the FP64 transposed operator (mixed)."""
    import torch
    L = nat.lib()
    n = bem.n
    s = nat.stream_ptr()
    prec = bem._cprec
    scr = torch.empty(int(L.bem200_bem_solve_T_workspace_size(prec, n, npol)), dtype=torch.uint8, device=bem.dev)
    lam = torch.empty_like(w)

    def sT(v, out):
        nat.call("bem200_bem_solve_T", prec, _engine(bem), n, npol, nat.ptr(bem._ws), nat.ptr(v), bem._eps_mode,
                 bem._e1p, bem._e2p, nat.ptr(bem._nvec), bem.k, nat.ptr(out), nat.ptr(scr), s)
    sT(w, lam)
    if prec == 0:
        return lam, 0
    G = bem._G128
    ascr = torch.empty(int(L.bem200_bem_apply_T_workspace_size(n, npol)), dtype=torch.uint8, device=bem.dev)
    r = torch.empty_like(w)
    d = torch.empty_like(w)
    wn = float(torch.linalg.vector_norm(w))
    for it in range(1, maxit + 1):
        nat.call("bem200_bem_apply_T", n, npol, *[nat.ptr(m) for m in G], bem._eps_mode, bem._e1p, bem._e2p,
                 nat.ptr(bem._nvec), bem.k, nat.ptr(lam), nat.ptr(w), nat.ptr(r), nat.ptr(ascr), s)
        rn = float(torch.linalg.vector_norm(r))
        if rn <= tol * wn:
            return lam, it
        sT(r, d)
        lam += d
    raise RuntimeError("transposed solve: refinement left the residual at {:.3e} (tol {:.1e})".format(rn / wn, tol))


def _engine(bem):
    from .bem import _ENGINES
    return _ENGINES[bem.engine]


def extinction_vertex_vjp(bem, exc, enei, weights=None):
    """Extinction of the plane wave ``exc`` at ``enei`` and the gradient of
    sum_q weights_q ext_q over every vertex coordinate (the vertex array of
    ``vertex_array(bem.p)``), from one solve and one transposed solve with
    the wavelength's factors.  Returns (ext (npol,), grad (nvert, 3))."""
    import torch
    p = bem.p
    g = bem.g
    bem.init(enei)
    npol = exc.pol.shape[0]
    if npol > 4:
        raise ValueError("extinction_vertex_vjp: at most 4 polarisations")
    wts = np.ones(npol) if weights is None else np.asarray(weights, dtype=float).reshape(npol)
    dev = bem.dev
    V = torch.as_tensor(vertex_array(p), dtype=torch.float64, device=dev).requires_grad_(True)
    geo = face_geometry(p, V)
    # the solution for the plane wave (device right-hand side)
    bt, _ = exc.rhs_device(p, enei, bem._eps_mode, bem._e1p, bem._e2p, device=dev)
    W1, W2 = bem.solve_device(bt, npol)
    x = torch.cat([W1.reshape(-1), W2.reshape(-1)])
    b, w, km = _planewave_terms(p, exc, enei, geo["pos"], geo["nvec"], geo["area"])
    n = p.n
    z = (w.detach().reshape(2, n, 4 * npol) * x.reshape(2, n, 4 * npol)).sum(dim=(0, 1)).reshape(4, npol)
    zq = z[0] + z[1:].sum(dim=0)  # column q of the solution layout belongs to polarisation q
    ext = (float(np.real(4 * np.pi / km)) * torch.imag(zq)).cpu().numpy()
    # adjoint of the weighted functional
    scale = torch.as_tensor(np.tile(wts, 4), dtype=torch.complex128, device=dev)            # per column of 4p
    wsc = (w.detach().reshape(2, n, 4 * npol) * scale[None, None, :]).reshape(-1).contiguous()
    lam, _ = _transposed_solve(bem, wsc, npol, tol=bem.ir_tol)
    # lambda^T A_v x on the GPU
    grad = _operator_gradient(bem, npol, W1, W2, lam)
    # w_v^T x + lambda^T b_v by autograd, minus lambda^T A_v x, chained to V
    s_pw = (w.reshape(2, n, 4 * npol) * scale[None, None, :] * x.reshape(2, n, 4 * npol)).sum() + (lam * b).sum()
    pref = float(np.real(4 * np.pi / km))
    outs = [geo["pos"], geo["nvec"], geo["area"], geo["tvec1"], geo["tvec2"], geo["nodes"]]
    gs = torch.autograd.grad(pref * torch.imag(s_pw), outs, allow_unused=True)
    cot = []
    for o, gpw, gk in zip(outs, gs, grad):
        c = -pref * torch.imag(gk).reshape(o.shape)
        cot.append(c if gpw is None else c + gpw)
    (gV,) = torch.autograd.grad(outs, [V], grad_outputs=cot)
    return ext, gV.detach().cpu().numpy()


def _operator_gradient(bem, npol, W1, W2, lam):
    """Complex cotangents of lambda^T A x over (pos, nvec, area, tvec1,
    tvec2, face nodes), from bem200_shape_gradient."""
    import torch
    g = bem.g
    r = g.refined
    n = bem.n
    dev = bem.dev
    L = nat.lib()
    nref = r.nref
    # refined rows of every column (CSC)
    key = r.col[:nref].long() * n + r.row[:nref].long()
    order = torch.argsort(key)
    csc_row = r.row[:nref][order].contiguous()
    counts = torch.bincount(r.col[:nref].long(), minlength=n)
    col_ptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    col_ptr[1:] = torch.cumsum(counts, 0)
    ks = g.wavenumbers(bem.enei)
    kmat = (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])
    blk = g._blk_mat([(0, 0), (1, 0), (1, 1), (0, 1)])
    grad = torch.zeros(40 * n, dtype=torch.complex128, device=dev)
    scr = torch.empty(int(L.bem200_shape_gradient_workspace_size(n, nref, g.order)), dtype=torch.uint8, device=dev)
    nat.call("bem200_shape_gradient", n, npol, g.npart, nat.ptr(g.pid), nat.ptr(blk), len(ks),
             ctypes.cast(kmat, ctypes.c_void_p), bem.k, bem._eps_mode, bem._e1p, bem._e2p, nat.ptr(g.closed_mask),
             nat.ptr(g.pos), nat.ptr(g.nvec), nat.ptr(g.tvec1), nat.ptr(g.tvec2), nat.ptr(g.area), nat.ptr(g.nodes),
             nat.ptr(g.face_kind), nat.ptr(g.rules), g.n28, g.n3, g.n4, nref, nat.ptr(r.row_ptr), nat.ptr(r.row),
             nat.ptr(r.col), nat.ptr(r.kind), nat.ptr(col_ptr), nat.ptr(csc_row), g.order, nat.ptr(r.g), nat.ptr(r.f),
             nat.ptr(g.corr), nat.ptr(W1), nat.ptr(W2), nat.ptr(lam), nat.ptr(grad), nat.ptr(scr), nat.stream_ptr())
    return (grad[:3 * n], grad[3 * n:6 * n], grad[6 * n:7 * n], grad[7 * n:10 * n], grad[10 * n:13 * n],
            grad[13 * n:])
