"""Derivatives of the extinction cross section with respect to a material's permittivity.

For one complex parameter the tangent (forward) sensitivity costs exactly one
more solve with the factors already built for the wavelength, the same as an
adjoint solve.  With A(eps) x = b the BEM system (b, the plane wave in the
embedding medium, does not depend on the particle's material):

    dx/deps = -A^-1 (dA/deps x),
    dA/deps x = A(M', e) x + A(M, e') x - A(M, 0) x,

because the operator is bilinear in the matrices M = (G1, G2, H1, H2) and the
per-face permittivities e.  M' = dM/dk dk/deps comes from the derivative
assembly kernel (bem200_green_assemble_dk), e' is 1 on the face sides that
belong to the material, dk/deps = k0 / (2 sqrt(eps)).  The extinction is
ext = 4 pi / k Im(z) with z = pol* . e_far(dir) linear in x, so for
eps = u + i v:  d ext/du = 4 pi / k Im(z'),  d ext/dv = 4 pi / k Re(z').

``ExtinctionEps`` wraps this as a torch.autograd.Function of (Re eps, Im eps).
The reference has no gradients; it is checked against central finite
differences of the solver (tests/test_adjoint_gpu.py).
"""
import ctypes

import numpy as np

from . import _native as nat


def _torch():
    import torch
    return torch


def _pe(exc, p, enei, W1, W2):
    """z_i = pol_i* . e_far(dir_i) for each polarisation (device W1, W2)."""
    torch = _torch()
    from .planewave import _face_tensors, _on_side
    npol = exc.pol.shape[0]
    dev = W1.device
    km = complex(np.asarray(p.eps[exc.medium - 1](enei)[1]).ravel()[0])
    k0 = 2 * np.pi / enei
    pos, _, area = _face_tensors(p, dev)
    side = _on_side(p, exc.medium, dev)
    dirs = torch.as_tensor(np.ascontiguousarray(exc.dir), device=dev)
    e = torch.empty((npol, 3, npol), dtype=torch.complex128, device=dev)
    h = torch.empty_like(e)
    kmh = (ctypes.c_double * 2)(km.real, km.imag)
    nat.call("bem200_farfield", p.n, npol, npol, nat.ptr(dirs), nat.ptr(pos), nat.ptr(area), nat.ptr(side), kmh, k0,
             nat.ptr(W1), nat.ptr(W2), nat.ptr(e), nat.ptr(h), nat.stream_ptr())
    e = e.cpu().numpy()
    return np.array([np.sum(np.conj(exc.pol[i]) * e[i, :, i]) for i in range(npol)]), km


def extinction_eps_gradient(bem, exc, enei, material):
    """Extinction and its gradient with respect to (Re eps, Im eps) of
    ``material`` (1-based index into p.eps) at wavelength ``enei``.

    ``bem`` is a BEMRet (fp64 or mixed).  Returns (ext (npol,), grad
    (npol, 2)).  Cost: the solve, three operator applications, one derivative
    assembly and one more solve with the same factors."""
    torch = _torch()
    p = bem.p
    n = p.n
    g = bem.g
    dev = bem.dev
    L = nat.lib()
    s = nat.stream_ptr()
    bem.init(enei)
    bt, npol = exc.rhs_device(p, enei, bem._eps_mode, bem._e1p, bem._e2p, device=dev)
    W1, W2 = bem.solve_device(bt, npol)
    x = torch.cat([W1.reshape(-1), W2.reshape(-1)])
    z, km = _pe(exc, p, enei, W1, W2)
    ext = np.real(4 * np.pi / km * np.imag(z))
    # the matrices M at enei (the mixed solver keeps them; the fp64 one factored its copies)
    if bem._prec == 1:
        M = bem._G128
    else:
        M = [torch.empty((n, n), dtype=torch.complex128, device=dev) for _ in range(4)]
        g.bem_matrices(enei, dtype="c128", out=M)
    # M' = dM/dk dk/deps for the material's wavenumber
    ks = g.wavenumbers(enei)
    kmat = (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])
    blk = g._blk_mat([(0, 0), (1, 0), (1, 1), (0, 1)])
    r = g.refined
    Md = [torch.empty((n, n), dtype=torch.complex128, device=dev) for _ in range(4)]
    nat.call("bem200_green_assemble_dk", n, g.npart, nat.ptr(g.pid), nat.ptr(blk), len(ks),
             ctypes.cast(kmat, ctypes.c_void_p), int(material), nat.ptr(g.pos), nat.ptr(g.nvec), nat.ptr(g.area),
             r.nref, nat.ptr(r.row), nat.ptr(r.col), g.order, nat.ptr(r.g), nat.ptr(r.fn), *[nat.ptr(m) for m in Md], n,
             s)
    eps_m = complex(np.asarray(p.eps[material - 1](enei)[0]).ravel()[0])
    k0 = 2 * np.pi / enei
    dk = k0 / (2.0 * np.sqrt(eps_m))
    for m in Md:
        m.mul_(dk)
    # e' per face side, and the zero permittivity
    io = np.asarray(p.inout_faces)
    d1 = torch.as_tensor((io[:, 0] == material).astype(np.complex128), device=dev)
    d2 = torch.as_tensor((io[:, 1] == material).astype(np.complex128), device=dev)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    zp = ctypes.cast(zero, ctypes.c_void_p)
    scr = torch.empty(int(L.bem200_bem_apply_workspace_size(n, npol)), dtype=torch.uint8, device=dev)
    np_ = n * npol
    xb = x.data_ptr()
    w1p, w2p = ctypes.c_void_p(xb), ctypes.c_void_p(xb + 16 * 4 * np_)

    def apply(mats, mode, e1, e2, out):
        nat.call("bem200_bem_apply", n, npol, *[nat.ptr(m) for m in mats], mode, e1, e2, nat.ptr(bem._nvec), bem.k,
                 w1p, w2p, None, nat.ptr(out), nat.ptr(scr), s)

    r1 = torch.empty(8 * np_, dtype=torch.complex128, device=dev)
    r2 = torch.empty_like(r1)
    r3 = torch.empty_like(r1)
    apply(Md, bem._eps_mode, bem._e1p, bem._e2p, r1)      # A(M', e) x
    apply(M, 1, nat.ptr(d1), nat.ptr(d2), r2)             # A(M, e') x
    apply(M, 0, zp, zp, r3)                               # A(M, 0) x
    rhs = -(r1 + r2 - r3)
    dW1, dW2 = bem.solve_device(rhs, npol)
    dz, _ = _pe(exc, p, enei, dW1, dW2)
    grad = np.stack([np.real(4 * np.pi / km * np.imag(dz)), np.real(4 * np.pi / km * np.real(dz))], axis=1)
    return ext, grad


class ExtinctionEps:
    """torch.autograd.Function: ext = ExtinctionEps.apply(eps_ri, bem, exc, enei, material)
    with eps_ri = (Re eps, Im eps) of the material as a float64 tensor (the
    value is used only to check that it matches the material at enei); the
    backward pass returns d ext / d (Re eps, Im eps)."""

    @staticmethod
    def apply(eps_ri, bem, exc, enei, material):
        torch = _torch()

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, e):
                ext, grad = extinction_eps_gradient(bem, exc, enei, material)
                ctx.save_for_backward(torch.as_tensor(grad, dtype=torch.float64))
                return torch.as_tensor(ext, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gout):
                (grad,) = ctx.saved_tensors
                return (gout.to(grad.dtype).reshape(-1, 1) * grad).sum(dim=0).to(gout.device)

        return _F.apply(eps_ri)
