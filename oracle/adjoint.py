"""Oracle: transposed BEM solve and reverse-mode derivatives of the extinction.

Test infrastructure only (see ``oracle/__init__.py``).  The reference has no
gradients; this module is the CPU specification that a reverse-mode GPU
adjoint follows, checked here by the adjoint identities and against the
tangent (forward-mode) derivatives and finite differences of the full solve.

Pairings are bilinear (no conjugation): for the solve S = A^-1 of
``oracle.bem.bem_solve`` (equation space (phi, a, alpha, De) -> unknowns
(sig1, sig2, h1, h2)), ``bem_solve_T`` applies S^T = A^-T, so that
<S^T u, v> = <u, S v>.  With the extinction functional z = w^T x and
A x = b, a derivative along any geometry direction is

    dz = dw^T x + lambda^T (db - dA x),     lambda = A^-T w,

one transposed solve for every direction (``reverse_directional``).
"""
import numpy as np
from scipy.linalg import lu_solve

from . import bem as obem
from . import farfield as off
from .pipeline import OracleBEM


def _L(L, x):
    return obem._apply_L(L, x)


def _nlift(nv, x):
    """(n, p) -> (n, 3, p): n_c x."""
    return nv[:, :, None] * x[:, None, :]


def _ndot(nv, y):
    """(n, 3, p) -> (n, p): sum_c n_c y_c."""
    return np.einsum("ij,ijk->ik", nv, y)


def bem_solve_T(st, gs1, gs2, gh1, gh2):
    """S^T applied to unknown-space cotangents (sig1, sig2 (n, p); h1, h2
    (n, 3, p)): returns (phi, a, alpha, De) cotangents.  Each step of
    ``oracle.bem.bem_solve`` transposed, in reverse order: G^-T and Sigma^-T
    are LU solves with trans=1, Delta^-T uses the Delta factors, Sigma1^T is
    the transposed matrix, and the per-face eps and normal products are
    their own transposes."""
    n = st.n
    k, nv = st.k, st.nvec

    def ls_T(lu, b):
        return lu_solve(lu, b.reshape(n, -1), trans=1, check_finite=False).reshape(b.shape)

    L = st.L1 - st.L2
    # sig1 = G1^-1 (sig2' + phi), h1 = G1^-1 (h2' + a), sig2 = G2^-1 sig2', h2 = G2^-1 h2'
    us1 = ls_T(st.G1_lu, gs1)
    uh1 = ls_T(st.G1_lu, gh1)
    b_sig2p = us1 + ls_T(st.G2_lu, gs2)
    b_h2p = uh1 + ls_T(st.G2_lu, gh2)
    b_phi = us1.copy()
    b_a = uh1.copy()
    # h2' = Delta^-1 (ik n (L sig2') + alpha_m)
    w = ls_T(st.Delta_lu, b_h2p)
    b_alpham = w.copy()
    b_sig2p = b_sig2p + 1j * k * _L(L, _ndot(nv, w))
    # sig2' = Sigma^-1 (De_m + ik n.(L Delta^-1 alpha_m))
    v = ls_T(st.Sigma_lu, b_sig2p)
    b_Dem = v
    b_alpham = b_alpham + ls_T(st.Delta_lu, _L(L, _nlift(nv, 1j * k * v)))
    # De_m = De - Sigma1 L1 phi + ik n.(L1 a)
    b_De = b_Dem.copy()
    b_phi = b_phi - _L(st.L1, st.Sigma1.T @ b_Dem)
    b_a = b_a + 1j * k * _L(st.L1, _nlift(nv, b_Dem))
    # alpha_m = alpha - Sigma1 a + ik n (L1 phi)
    b_alpha = b_alpham.copy()
    b_a = b_a - (st.Sigma1.T @ b_alpham.reshape(n, -1)).reshape(b_alpham.shape)
    b_phi = b_phi + 1j * k * _L(st.L1, _ndot(nv, b_alpham))
    return b_phi, b_a, b_alpha, b_De


def bem_operator_T(G1, G2, H1, H2, eps1, eps2, nvec, enei, lphi, la, lalpha, lDe):
    """A^T of ``oracle.bem.bem_operator``: equation-space cotangents ->
    (sig1, sig2, h1, h2) cotangents.  Every product is with a transposed
    matrix; eps (at the source point in A) is applied after it here."""
    k = 2 * np.pi / enei
    e1 = np.asarray(eps1).reshape(-1, 1) if np.ndim(eps1) else eps1
    e2 = np.asarray(eps2).reshape(-1, 1) if np.ndim(eps2) else eps2
    e1h = e1[:, :, None] if np.ndim(e1) else e1
    e2h = e2[:, :, None] if np.ndim(e2) else e2
    n = G1.shape[0]

    def mt(M, x):
        return (M.T @ x.reshape(n, -1)).reshape(x.shape)

    na = _ndot(nvec, lalpha)
    nD = _nlift(nvec, lDe)
    s1 = mt(G1, lphi) - 1j * k * e1 * mt(G1, na) + e1 * mt(H1, lDe)
    s2 = -mt(G2, lphi) + 1j * k * e2 * mt(G2, na) - e2 * mt(H2, lDe)
    h1 = mt(G1, la) + mt(H1, lalpha) - 1j * k * e1h * mt(G1, nD)
    h2 = -mt(G2, la) - mt(H2, lalpha) + 1j * k * e2h * mt(G2, nD)
    return s1, s2, h1, h2


def extinction_weights(cp, enei, pol, dirs, medium=1):
    """w with z_i = sum(w_sig1 s1 + w_sig2 s2 + w_h1 . h1 + w_h2 . h2)[:, i],
    z_i = conj(pol_i) . e_far(dir_i) of ``oracle.farfield.extinction``.
    Returns (w_s1, w_s2 (n, p), w_h1, w_h2 (n, 3, p))."""
    pol = np.atleast_2d(pol)
    dirs = np.atleast_2d(dirs).astype(float)
    k = complex(np.asarray(cp.eps[medium - 1](enei)[1]).ravel()[0])
    k0 = 2 * np.pi / enei
    p = pol.shape[0]
    io = cp.inout_faces
    ws = [np.zeros((cp.n, p), dtype=complex) for _ in range(2)]
    wh = [np.zeros((cp.n, 3, p), dtype=complex) for _ in range(2)]
    for i in range(p):
        phase = np.exp(-1j * k * (cp.pos @ dirs[i])) * cp.area
        pc = np.conj(pol[i])
        for side in range(2):
            on = (io[:, side] == medium).astype(float)
            ws[side][:, i] = -1j * k * np.dot(pc, dirs[i]) * phase * on
            wh[side][:, :, i] = 1j * k0 * (phase * on)[:, None] * pc[None, :]
    return ws[0], ws[1], wh[0], wh[1]


def _pair(a, b):
    return sum(np.sum(x * y, axis=tuple(range(x.ndim - 1))) for x, y in zip(a, b))


def _state(cp, enei, pol, dirs):
    ob = OracleBEM(cp)
    G1, G2, H1, H2 = ob.matrices(enei)
    e1, e2 = cp.eps1(enei), cp.eps2(enei)
    st = obem.bem_init(G1, G2, H1, H2, e1, e2, cp.nvec, enei, con01_zero=True)
    rhs = obem.excitation(st, off.planewave_potential(cp, pol, dirs, enei), e1, e2)
    return (G1, G2, H1, H2, e1, e2), st, rhs


def reverse_directional(cp, enei, pol, dirs, directions, h=1e-4):
    """Extinction and its derivatives along vertex ``directions`` (K, nvert, 3)
    of the vertex space of mnpbem_b200.shape, by one transposed solve:
    dz_k = dw_k^T x + lambda^T (db_k - dA_k x), lambda = A^-T w.  The
    geometry derivatives dw, db, dA x are central differences (step h) of
    the oracle's assembly at v +- h D_k, as in the GPU tangent method.
    Returns (ext (p,), dext (K, p), lambda)."""
    from mnpbem_b200.shape import perturbed
    pol = np.atleast_2d(pol)
    mats, st, rhs = _state(cp, enei, pol, dirs)
    x = obem.bem_solve(st, *rhs)                    # sig1, sig2, h1, h2
    w = extinction_weights(cp, enei, pol, dirs)
    z = _pair(w, x)
    lam = bem_solve_T(st, *w)
    k = complex(np.asarray(cp.eps[0](enei)[1]).ravel()[0])
    ext = np.real(4 * np.pi / k * np.imag(z))
    D = np.asarray(directions, dtype=float)
    D = D[None] if D.ndim == 2 else D
    dext = []
    for d in D:
        side = []
        for s in (1.0, -1.0):
            q = perturbed(cp, s * h * d)
            (G1, G2, H1, H2, e1, e2), stq, rhsq = _state(q, enei, pol, dirs)
            Ax = obem.bem_operator(G1, G2, H1, H2, e1, e2, q.nvec, enei, x[0], x[1], x[2], x[3])
            wq = extinction_weights(q, enei, pol, dirs)
            side.append((Ax, rhsq, _pair(wq, x)))
        (Ap, bp, zp), (Am, bm, zm) = side
        # equation-space order of A x / b: (phi, a, alpha, De)
        r = [((bp[i] - bm[i]) - (Ap[i] - Am[i])) / (2 * h) for i in range(4)]
        dz = (zp - zm) / (2 * h) + _pair(lam, r)
        dext.append(np.real(4 * np.pi / k * np.imag(dz)))
    return ext, np.array(dext), lam


def tangent_directional(cp, enei, pol, dirs, directions, h=1e-4):
    """The same derivatives by one forward (tangent) solve per direction:
    dx = A^-1 (db - dA x)."""
    from mnpbem_b200.shape import perturbed
    pol = np.atleast_2d(pol)
    mats, st, rhs = _state(cp, enei, pol, dirs)
    x = obem.bem_solve(st, *rhs)
    w = extinction_weights(cp, enei, pol, dirs)
    k = complex(np.asarray(cp.eps[0](enei)[1]).ravel()[0])
    dext = []
    for d in directions:
        side = []
        for s in (1.0, -1.0):
            q = perturbed(cp, s * h * d)
            (G1, G2, H1, H2, e1, e2), _, rhsq = _state(q, enei, pol, dirs)
            Ax = obem.bem_operator(G1, G2, H1, H2, e1, e2, q.nvec, enei, x[0], x[1], x[2], x[3])
            side.append((Ax, rhsq, _pair(extinction_weights(q, enei, pol, dirs), x)))
        (Ap, bp, zp), (Am, bm, zm) = side
        r = [((bp[i] - bm[i]) - (Ap[i] - Am[i])) / (2 * h) for i in range(4)]
        dx = obem.bem_solve(st, *r)
        dz = (zp - zm) / (2 * h) + _pair(w, dx)
        dext.append(np.real(4 * np.pi / k * np.imag(dz)))
    return np.array(dext)
