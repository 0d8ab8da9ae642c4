"""Plane-wave excitation, far fields and cross sections (host side).

Mirrors ``PlaneWaveRet`` (mnpbem/simulation/planewave_ret.py:17) and
``SpectrumRet`` (mnpbem/spectrum/spectrum_ret.py:136): ``potential(p, enei)``
gives the vector potentials on both sides of every face, ``extinction``
uses the optical theorem and ``scattering`` integrates the Poynting vector
over the 256-direction unit sphere.  These are O(N) per polarisation and run
on the host, as in the reference.
"""
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


class CompStruct:
    """Attribute container with dict-style access (reference compgreen_stat.py:1154)."""

    def __init__(self, p, enei, **fields):
        self.p = p
        self.enei = enei
        for k, v in fields.items():
            setattr(self, k, v)

    def set(self, **fields):
        for k, v in fields.items():
            setattr(self, k, v)
        return self

    def get(self, name, default=None):
        return getattr(self, name, default)

    def __getitem__(self, name):
        return getattr(self, name)

    def __contains__(self, name):
        return hasattr(self, name)


def _pinfty():
    d = np.load(os.path.join(_DATA, "pinfty256.npz"))
    return d["nvec"], d["area"]


class SpectrumRet:
    """Far fields on a discretised unit sphere (default: the 256-direction sphere)."""

    def __init__(self, pinfty=None, medium=1):
        self.medium = medium
        if pinfty is None:
            self.nvec, self.area = _pinfty()
        else:
            self.nvec = np.atleast_2d(np.asarray(pinfty.nvec if hasattr(pinfty, "nvec") else pinfty, dtype=float))
            self.area = (np.asarray(pinfty.area) if hasattr(pinfty, "area")
                         else np.full(len(self.nvec), 4 * np.pi / len(self.nvec)))
        self.ndir = len(self.nvec)

    def farfield(self, sig, direction=None):
        """e, h (ndir, 3, p) far-field amplitudes (spectrum_ret.py:231-392)."""
        dirs = self.nvec if direction is None else np.atleast_2d(np.asarray(direction, dtype=float))
        p = sig.p
        enei = sig.enei
        k = complex(np.asarray(p.eps[self.medium - 1](enei)[1]).ravel()[0])
        k0 = 2 * np.pi / enei
        phase = np.exp(-1j * k * (dirs @ p.pos.T)) * p.area
        io = p.inout_faces
        s1, s2, h1, h2 = (np.asarray(getattr(sig, name)) for name in ("sig1", "sig2", "h1", "h2"))
        if s1.ndim == 1:
            s1, s2, h1, h2 = s1[:, None], s2[:, None], h1[:, :, None], h2[:, :, None]
        npol = s1.shape[1]
        e = np.zeros((len(dirs), 3, npol), dtype=complex)
        h = np.zeros((len(dirs), 3, npol), dtype=complex)
        for side, s, hh in ((0, s1, h1), (1, s2, h2)):
            ind = np.flatnonzero(io[:, side] == self.medium)
            if len(ind) == 0:
                continue
            ph = phase[:, ind]
            phh = np.einsum("dn,ncp->dcp", ph, hh[ind])
            phs = ph @ s[ind]
            e += 1j * k0 * phh - 1j * k * dirs[:, :, None] * phs[:, None, :]
            h += 1j * k * np.cross(dirs[:, :, None], phh, axis=1)
        return e, h

    def scattering(self, sig):
        e, h = self.farfield(sig)
        dsca = 0.5 * np.real(np.einsum("dc,dcp->dp", self.nvec, np.cross(e, np.conj(h), axis=1)))
        sca = self.area @ dsca
        if sca.size == 1:
            return float(sca[0]), dsca[:, 0]
        return sca, dsca


def _on_side(p, medium, device):
    """(n, 2) int8 device mask: face side s faces the embedding medium."""
    import torch
    key = (id(p), medium, str(device))
    cache = getattr(p, "_b200_side_cache", None)
    if cache is not None and cache[0] == key:
        return cache[1]
    io = np.asarray(p.inout_faces)
    m = torch.as_tensor(np.ascontiguousarray((io == medium).astype(np.int8)), device=device)
    p._b200_side_cache = (key, m)
    return m


def _face_tensors(p, device):
    import torch
    cache = getattr(p, "_b200_face_cache", None)
    if cache is not None and cache[0] == str(device):
        return cache[1]
    f64 = dict(dtype=torch.float64, device=device)
    t = (torch.as_tensor(np.ascontiguousarray(p.pos), **f64), torch.as_tensor(np.ascontiguousarray(p.nvec), **f64),
         torch.as_tensor(np.ascontiguousarray(p.area), **f64))
    p._b200_face_cache = (str(device), t)
    return t


class PlaneWaveRet:
    """Plane wave exp(i k dir.r) with polarisation pol (one row per excitation)."""

    def __init__(self, pol, dir, medium=1, pinfty=None, **options):
        if pol is None or dir is None:
            raise ValueError("PlaneWaveRet: 'pol' and 'dir' are required")
        self.pol = np.atleast_2d(np.asarray(pol, dtype=float))
        self.dir = np.atleast_2d(np.asarray(dir, dtype=float))
        if self.pol.shape[1] != 3 or self.dir.shape[1] != 3:
            raise ValueError("PlaneWaveRet: pol and dir must have shape (npol, 3)")
        self.medium = options.get("medium", medium)
        self.spec = SpectrumRet(pinfty, medium=self.medium)

    def potential(self, p, enei):
        """a1, a1p, a2, a2p on the faces touching the embedding medium
        (planewave_ret.py:257-361)."""
        if not np.allclose(np.sum(self.pol * self.dir, axis=1), 0):
            raise ValueError("PlaneWaveRet: polarisation and direction must be orthogonal")
        eps_val = p.eps[self.medium - 1](enei)[0]
        k0 = 2 * np.pi / enei
        k = k0 * np.sqrt(eps_val)
        npol = self.pol.shape[0]
        io = p.inout_faces
        exc = CompStruct(p, enei)
        for side, name in ((0, "1"), (1, "2")):
            a = np.zeros((p.n, 3, npol), dtype=complex)
            ap = np.zeros((p.n, 3, npol), dtype=complex)
            ind = np.flatnonzero(io[:, side] == self.medium)
            for i in range(npol):
                if len(ind):
                    ph = np.exp(1j * k * p.pos[ind] @ self.dir[i]) / (1j * k0)
                    a[ind, :, i] = ph[:, None] * self.pol[i]
                    ap[ind, :, i] = (1j * k * (p.nvec[ind] @ self.dir[i]))[:, None] * ph[:, None] * self.pol[i]
            if npol == 1:
                a, ap = a[:, :, 0], ap[:, :, 0]
            exc.set(**{"a" + name: a, "a" + name + "p": ap})
        return exc

    __call__ = potential

    def field(self, p, enei, inout=1):
        """Electric and magnetic field of the plane wave at the faces whose
        side ``inout`` (1 inside, 2 outside) touches the embedding medium:
        e = exp(i k dir.r) pol, h = n_b dir x e (reference
        planewave_ret.py:157-255).  Returns CompStruct(e, h), (n, 3[, npol])."""
        if not np.allclose(np.sum(self.pol * self.dir, axis=1), 0):
            raise ValueError("PlaneWaveRet: polarisation and direction must be orthogonal")
        eps_val = p.eps[self.medium - 1](enei)[0]
        nb = np.sqrt(eps_val)
        k0 = 2 * np.pi / enei
        k = k0 * nb
        npol = self.pol.shape[0]
        ind = np.flatnonzero(np.asarray(p.inout_faces)[:, inout - 1] == self.medium)
        e = np.zeros((p.n, 3, npol), dtype=complex)
        h = np.zeros((p.n, 3, npol), dtype=complex)
        for i in range(npol):
            if len(ind):
                ph = np.exp(1j * k * p.pos[ind] @ self.dir[i]) / (1j * k0)
                e[ind, :, i] = 1j * k0 * ph[:, None] * self.pol[i]
            h[:, :, i] = nb * np.cross(np.tile(self.dir[i], (p.n, 1)), e[:, :, i])
        if npol == 1:
            e, h = e[:, :, 0], h[:, :, 0]
        return CompStruct(p, enei, e=e, h=h)

    def rhs_device(self, p, enei, eps_mode, e1p, e2p, device="cuda"):
        """The BEM right-hand side of this plane wave directly on the device
        (8 n npol complex128, layout of BEMRet.rhs): potential() fused with the
        excitation of BEMRet (planewave_ret.py:257-361, bem_ret.py:1360-1429).
        eps_mode / e1p / e2p: the eps arguments of the C ABI."""
        import ctypes
        import torch
        from . import _native as nat
        if not np.allclose(np.sum(self.pol * self.dir, axis=1), 0):
            raise ValueError("PlaneWaveRet: polarisation and direction must be orthogonal")
        npol = self.pol.shape[0]
        eps_val = complex(np.asarray(p.eps[self.medium - 1](enei)[0]).ravel()[0])
        k0 = 2 * np.pi / enei
        km = k0 * np.sqrt(eps_val)
        pos, nvec, _ = _face_tensors(p, device)
        side = _on_side(p, self.medium, device)
        b = torch.empty(8 * p.n * npol, dtype=torch.complex128, device=device)
        pol = (ctypes.c_double * (3 * npol))(*self.pol.ravel())
        dirs = (ctypes.c_double * (3 * npol))(*self.dir.ravel())
        kmh = (ctypes.c_double * 2)(km.real, km.imag)
        nat.call("bem200_planewave_rhs", p.n, npol, nat.ptr(pos), nat.ptr(nvec), nat.ptr(side), pol, dirs, kmh, k0,
                 eps_mode, e1p, e2p, nat.ptr(b), nat.stream_ptr())
        return b, npol

    def cross_sections_device(self, p, enei, W1, W2):
        """Extinction and scattering from device solutions W1 = [sig1 | h1],
        W2 = [sig2 | h2] (n x 4 npol): far fields on the GPU, the O(ndir)
        sums on the host.  Returns (ext (npol,), sca (npol,), dsca (ndir, npol))."""
        import ctypes
        import torch
        from . import _native as nat
        npol = self.pol.shape[0]
        dev = W1.device
        km = complex(np.asarray(p.eps[self.medium - 1](enei)[1]).ravel()[0])
        k0 = 2 * np.pi / enei
        pos, _, area = _face_tensors(p, dev)
        side = _on_side(p, self.medium, dev)
        spec = self.spec
        if getattr(spec, "_dev_dirs", None) is None or spec._dev_dirs.device != dev:
            spec._dev_dirs = torch.as_tensor(np.ascontiguousarray(np.vstack([spec.nvec, self.dir])), device=dev)
        nd = spec._dev_dirs.shape[0]
        e = torch.empty((nd, 3, npol), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        kmh = (ctypes.c_double * 2)(km.real, km.imag)
        nat.call("bem200_farfield", p.n, npol, nd, nat.ptr(spec._dev_dirs), nat.ptr(pos), nat.ptr(area), nat.ptr(side),
                 kmh, k0, nat.ptr(W1), nat.ptr(W2), nat.ptr(e), nat.ptr(h), nat.stream_ptr())
        e, h = e.cpu().numpy(), h.cpu().numpy()
        ns = spec.ndir
        dsca = 0.5 * np.real(np.einsum("dc,dcp->dp", spec.nvec, np.cross(e[:ns], np.conj(h[:ns]), axis=1)))
        nb = np.real(np.sqrt(complex(np.asarray(p.eps[self.medium - 1](enei)[0]).ravel()[0])))
        sca = (spec.area @ dsca) / (0.5 * nb)
        einc = e[ns:]
        pe = np.array([np.sum(np.conj(self.pol[i]) * einc[i, :, i]) for i in range(npol)])
        ext = np.real(4 * np.pi / km * np.imag(pe))
        return ext, sca, dsca / (0.5 * nb)

    def extinction(self, sig):
        """Optical theorem (planewave_ret.py:437-504)."""
        e, _ = self.spec.farfield(sig, self.dir)
        k = complex(np.asarray(sig.p.eps[self.medium - 1](sig.enei)[1]).ravel()[0])
        npol = self.pol.shape[0]
        pe = np.array([np.sum(np.conj(self.pol[i]) * e[i, :, i if e.shape[2] > 1 else 0]) for i in range(npol)])
        ext = np.real(4 * np.pi / k * np.imag(pe))
        return float(ext[0]) if npol == 1 else ext

    def scattering(self, sig):
        """(sca, dsca) normalised to the incoming power 0.5 n_b (planewave_ret.py:391-435)."""
        sca, dsca = self.spec.scattering(sig)
        nb = np.real(np.sqrt(complex(np.asarray(sig.p.eps[self.medium - 1](sig.enei)[0]).ravel()[0])))
        return sca / (0.5 * nb), dsca / (0.5 * nb)

    def absorption(self, sig):
        return self.extinction(sig) - self.scattering(sig)[0]
