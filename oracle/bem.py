"""Oracle: dense retarded BEM (BEMRet) in complex128 with scipy LAPACK.

Test infrastructure only (see ``oracle/__init__.py``).
"""
import numpy as np
from scipy.linalg import lu_factor, lu_solve


class BEMState:
    pass


def _diag_or_scalar(v):
    v = np.asarray(v)
    if np.allclose(v, v[0]):
        return v[0]
    return v


def bem_init(G1, G2, H1, H2, eps1, eps2, nvec, enei, con01_zero=True):
    """Sigma / Delta build of the dense retarded BEM.

    Sigma_i = H_i G_i^-1, Delta = Sigma1 - Sigma2,
    Sigma = Sigma1 L1 - Sigma2 L2 + k^2 (L Delta^-1 o n n^T) L, L = L1 - L2,
    with L_i = eps_i (scalar or diagonal; the cross-connected non-uniform case
    L_i = G_i eps_i G_i^-1 is not covered).
    Reference: mnpbem/bem/bem_ret.py:357-525 (MATLAB BEM/@bemret/private/initmat.m:5-72).
    """
    if not con01_zero and np.ndim(_diag_or_scalar(eps1)) > 0:
        raise NotImplementedError("cross-connected regions with non-uniform eps")
    st = BEMState()
    st.k = 2 * np.pi / enei
    st.nvec = nvec
    st.eps1 = _diag_or_scalar(eps1)
    st.eps2 = _diag_or_scalar(eps2)
    n = G1.shape[0]
    st.G1_lu = lu_factor(G1, check_finite=False)
    st.G2_lu = lu_factor(G2, check_finite=False)
    G1i = lu_solve(st.G1_lu, np.eye(n), check_finite=False)
    G2i = lu_solve(st.G2_lu, np.eye(n), check_finite=False)
    st.L1, st.L2 = st.eps1, st.eps2
    st.Sigma1 = H1 @ G1i
    Sigma2 = H2 @ G2i
    st.Delta_lu = lu_factor(st.Sigma1 - Sigma2, check_finite=False)
    Deltai = lu_solve(st.Delta_lu, np.eye(n), check_finite=False)
    nn = nvec @ nvec.T
    L = st.L1 - st.L2
    if np.ndim(L) == 0:
        Sigma = st.Sigma1 * st.L1 - Sigma2 * st.L2 + st.k ** 2 * L * (Deltai * nn) * L
    else:
        Sigma = (st.Sigma1 * st.L1[None, :] - Sigma2 * st.L2[None, :]
                 + st.k ** 2 * ((L[:, None] * Deltai) * nn) * L[None, :])
    st.Sigma_lu = lu_factor(Sigma, check_finite=False)
    st.n = n
    return st


def excitation(st, exc, eps1f, eps2f):
    """phi, a, alpha, De from the potentials of an excitation (Eqs. 10, 11, 15, 18).

    Reference: mnpbem/bem/bem_ret.py:1360-1429 (MATLAB excitation.m:21-29).
    ``exc`` holds (n,[p]) / (n,3,[p]) arrays for phi1, phi1p, a1, a1p, phi2,
    phi2p, a2, a2p (missing = 0); ``eps1f``/``eps2f`` are per-face eps.
    """
    n = st.n
    p = _npol(exc)
    z1 = np.zeros((n, p), dtype=complex)
    z3 = np.zeros((n, 3, p), dtype=complex)

    def get(name, z):
        v = exc.get(name, None)
        if v is None or (np.isscalar(v) and v == 0):
            return z
        v = np.asarray(v, dtype=complex)
        return v.reshape(z.shape)

    phi1, phi1p, phi2, phi2p = (get(k, z1) for k in ("phi1", "phi1p", "phi2", "phi2p"))
    a1, a1p, a2, a2p = (get(k, z3) for k in ("a1", "a1p", "a2", "a2p"))
    k = st.k
    nv = st.nvec
    e1 = eps1f[:, None]
    e2 = eps2f[:, None]
    phi = phi2 - phi1
    a = a2 - a1
    alpha = (a2p - a1p) - 1j * k * (nv[:, :, None] * (phi2 * e2)[:, None, :]
                                    - nv[:, :, None] * (phi1 * e1)[:, None, :])
    De = (e2 * phi2p - e1 * phi1p) - 1j * k * (np.einsum("ij,ijk->ik", nv, a2) * e2
                                                - np.einsum("ij,ijk->ik", nv, a1) * e1)
    return phi, a, alpha, De


def _npol(exc):
    for key in ("a1", "a2", "a1p", "a2p"):
        v = exc.get(key, None)
        if isinstance(v, np.ndarray) and v.ndim == 3:
            return v.shape[2]
    for key in ("phi1", "phi2", "phi1p", "phi2p"):
        v = exc.get(key, None)
        if isinstance(v, np.ndarray) and v.ndim == 2:
            return v.shape[1]
    return 1


def _apply_L(L, x):
    if np.ndim(L) == 0:
        return L * x
    return L.reshape((-1,) + (1,) * (x.ndim - 1)) * x


def bem_solve(st, phi, a, alpha, De):
    """Eqs. (19, 20) of Garcia de Abajo & Howie with the multi-RHS layout
    phi (n,p), a (n,3,p), alpha (n,3,p), De (n,p).

    Reference: mnpbem/bem/bem_ret.py:1754-1810 (npol > 1 branch; identical
    algebra to the npol = 1 branch :1709-1752; MATLAB mldivide.m:29-49).
    Returns sig1 (n,p), sig2 (n,p), h1 (n,3,p), h2 (n,3,p).
    """
    n = st.n
    p = phi.shape[1]
    k, nv = st.k, st.nvec

    def ls(lu, b):
        return lu_solve(lu, b.reshape(n, -1), check_finite=False).reshape(b.shape)

    L1phi = _apply_L(st.L1, phi)
    L1a = _apply_L(st.L1, a)
    S1a = (st.Sigma1 @ a.reshape(n, -1)).reshape(n, 3, p)
    alpha_m = alpha - S1a + 1j * k * (nv[:, :, None] * L1phi[:, None, :])
    De_m = De - st.Sigma1 @ L1phi + 1j * k * np.einsum("ij,ijk->ik", nv, L1a)
    L = st.L1 - st.L2
    inner = np.einsum("ij,ijk->ik", nv, _apply_L(L, ls(st.Delta_lu, alpha_m)))
    sig2 = ls(st.Sigma_lu, De_m + 1j * k * inner)
    h2 = ls(st.Delta_lu, 1j * k * (nv[:, :, None] * _apply_L(L, sig2)[:, None, :]) + alpha_m)
    sig1 = ls(st.G1_lu, sig2 + phi)
    h1 = ls(st.G1_lu, h2 + a)
    return sig1, ls(st.G2_lu, sig2), h1, ls(st.G2_lu, h2)


def bem_operator(G1, G2, H1, H2, eps1, eps2, nvec, enei, sig1, sig2, h1, h2):
    """Apply the full retarded BEM operator to (sig1, h1, sig2, h2):
    phi = G1 s1 - G2 s2, a = G1 h1 - G2 h2,
    alpha = H1 h1 - H2 h2 - ik n (G1 eps1 s1 - G2 eps2 s2),
    De = H1 eps1 s1 - H2 eps2 s2 - ik n.(G1 eps1 h1 - G2 eps2 h2).
    Reference: mnpbem/bem/bem_ret_iter.py:1362-1501 (_afun, eps applied at the
    source point).  Arrays carry a trailing polarisation axis.
    """
    k = 2 * np.pi / enei
    n = G1.shape[0]
    e1 = np.asarray(eps1).reshape(-1, 1) if np.ndim(eps1) else eps1
    e2 = np.asarray(eps2).reshape(-1, 1) if np.ndim(eps2) else eps2

    def mv(M, x):
        return (M @ x.reshape(n, -1)).reshape(x.shape)

    e1h = e1[:, :, None] if np.ndim(e1) else e1
    e2h = e2[:, :, None] if np.ndim(e2) else e2
    phi = mv(G1, sig1) - mv(G2, sig2)
    a = mv(G1, h1) - mv(G2, h2)
    alpha = mv(H1, h1) - mv(H2, h2) - 1j * k * nvec[:, :, None] * (mv(G1, e1 * sig1) - mv(G2, e2 * sig2))[:, None, :]
    De = mv(H1, e1 * sig1) - mv(H2, e2 * sig2) - 1j * k * np.einsum(
        "ij,ijk->ik", nvec, mv(G1, e1h * h1) - mv(G2, e2h * h2))
    return phi, a, alpha, De


def iter_solve(G1, G2, H1, H2, eps1, eps2, nvec, enei, phi, a, alpha, De, tol=1e-4, maxit=200, restart=None):
    """Unpreconditioned iterative solve of the BEM system, restating
    BEMRetIter.solve with precond=None (mnpbem/bem/bem_ret_iter.py:1636-1744):
    scipy GMRES (BEMIter._iter_solve, mnpbem/bem/bem_iter.py:86-90, restart
    defaulting to maxit) on x = pack(sig1, h1, sig2, h2) against
    b = pack(phi, a, De, alpha), column-major packing (:1196-1233), with
    the operator of ``bem_operator``.  Single polarisation.
    Returns sig1 (n,), sig2 (n,), h1 (n,3), h2 (n,3), iterations, relres."""
    import scipy.sparse.linalg as spl
    n = G1.shape[0]

    def pack(*arrs):
        return np.concatenate([np.asarray(v).reshape(n, -1).ravel(order="F") for v in arrs])

    def unpack_x(x):
        s1 = x[:n]
        h1 = x[n:4 * n].reshape(n, 3, order="F")
        s2 = x[4 * n:5 * n]
        h2 = x[5 * n:].reshape(n, 3, order="F")
        return s1, h1, s2, h2

    def mv(x):
        s1, h1, s2, h2 = unpack_x(x)
        ph, aa, al, de = bem_operator(G1, G2, H1, H2, eps1, eps2, nvec, enei, s1[:, None], s2[:, None],
                                      h1[:, :, None], h2[:, :, None])
        return pack(ph[:, 0], aa[:, :, 0], de[:, 0], al[:, :, 0])

    b = pack(phi[:, 0], a[:, :, 0], De[:, 0], alpha[:, :, 0])
    A = spl.LinearOperator((8 * n, 8 * n), matvec=mv, dtype=complex)
    count = []
    rs = restart if restart is not None else min(8 * n, maxit)
    x, flag = spl.gmres(A, b, rtol=tol, maxiter=maxit, restart=rs, callback=lambda rk: count.append(rk),
                        callback_type="pr_norm")
    relres = np.linalg.norm(mv(x) - b) / np.linalg.norm(b)
    s1, h1, s2, h2 = unpack_x(x)
    return s1, s2, h1, h2, len(count), relres
