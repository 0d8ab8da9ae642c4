"""Oracle: plane-wave potentials, far fields and cross sections (numpy).

Test infrastructure only (see ``oracle/__init__.py``).
"""
import numpy as np


def planewave_potential(cp, pol, dirs, enei, medium=1):
    """Vector potential a = exp(ik r.dir)/(ik0) pol and a' = ik (n.dir) a on the
    side of each face that touches ``medium``.
    Reference: mnpbem/simulation/planewave_ret.py:257-361 (MATLAB potential.m).
    Returns dict with a1, a1p, a2, a2p of shape (n, 3, p).
    """
    pol = np.atleast_2d(pol).astype(float)
    dirs = np.atleast_2d(dirs).astype(float)
    eps_val = cp.eps[medium - 1](enei)[0]
    k0 = 2 * np.pi / enei
    k = k0 * np.sqrt(eps_val)
    npol = pol.shape[0]
    io = cp.inout_faces
    out = {}
    for side, name in ((0, "1"), (1, "2")):
        a = np.zeros((cp.n, 3, npol), dtype=complex)
        ap = np.zeros((cp.n, 3, npol), dtype=complex)
        ind = np.flatnonzero(io[:, side] == medium)
        if len(ind):
            for i in range(npol):
                ph = np.exp(1j * k * cp.pos[ind] @ dirs[i]) / (1j * k0)
                a[ind, :, i] = ph[:, None] * pol[i]
                ap[ind, :, i] = (1j * k * (cp.nvec[ind] @ dirs[i]))[:, None] * ph[:, None] * pol[i]
        out["a" + name] = a
        out["a" + name + "p"] = ap
    return out


def farfield(cp, sig1, sig2, h1, h2, enei, dirs, medium=1):
    """Far-field amplitudes e, h (ndir, 3, p).
    Reference: mnpbem/spectrum/spectrum_ret.py:231-392 (Garcia de Abajo,
    Rev. Mod. Phys. 82, 209, Eq. 50)."""
    k = complex(np.asarray(cp.eps[medium - 1](enei)[1]).ravel()[0])
    k0 = 2 * np.pi / enei
    phase = np.exp(-1j * k * (dirs @ cp.pos.T)) * cp.area
    io = cp.inout_faces
    p = sig1.shape[1]
    e = np.zeros((len(dirs), 3, p), dtype=complex)
    h = np.zeros((len(dirs), 3, p), dtype=complex)
    for side, s, hh in ((0, sig1, h1), (1, sig2, h2)):
        ind = np.flatnonzero(io[:, side] == medium)
        if len(ind) == 0:
            continue
        ph = phase[:, ind]
        for ip in range(p):
            phh = ph @ hh[ind, :, ip]
            phs = ph @ s[ind, ip]
            e[:, :, ip] += 1j * k0 * phh - 1j * k * dirs * phs[:, None]
            h[:, :, ip] += 1j * k * np.cross(dirs, phh)
    return e, h


def extinction(cp, sig1, sig2, h1, h2, enei, pol, dirs, medium=1):
    """Optical theorem ext = 4 pi / k Im(conj(pol) . e_forward).
    Reference: mnpbem/simulation/planewave_ret.py:437-504."""
    pol = np.atleast_2d(pol)
    dirs = np.atleast_2d(dirs).astype(float)
    e, _ = farfield(cp, sig1, sig2, h1, h2, enei, dirs, medium)
    k = cp.eps[medium - 1](enei)[1]
    npol = pol.shape[0]
    pe = np.array([np.sum(np.conj(pol[i]) * e[i, :, i]) for i in range(npol)])
    return np.real(4 * np.pi / k * np.imag(pe))


def scattering(cp, sig1, sig2, h1, h2, enei, pinfty_nvec, pinfty_area, medium=1):
    """sca = sum_dir area * 0.5 Re(n.(E x H*)) / (0.5 n_b).
    Reference: mnpbem/spectrum/spectrum_ret.py:395-459 and
    mnpbem/simulation/planewave_ret.py:391-435."""
    e, h = farfield(cp, sig1, sig2, h1, h2, enei, pinfty_nvec, medium)
    p = e.shape[2]
    dsca = np.zeros((len(pinfty_nvec), p))
    for ip in range(p):
        pv = np.cross(e[:, :, ip], np.conj(h[:, :, ip]))
        dsca[:, ip] = 0.5 * np.real(np.sum(pinfty_nvec * pv, axis=1))
    sca = pinfty_area @ dsca
    nb = np.real(np.sqrt(cp.eps[medium - 1](enei)[0]))
    return np.asarray(sca / (0.5 * nb)).ravel()
