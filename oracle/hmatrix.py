"""Oracle: partially pivoted adaptive cross approximation -- TEST INFRASTRUCTURE.

Restates HMatrix._aca_block (mnpbem/greenfun/hmatrix.py:195-336) in numpy:
start at row 0; residual row -> pivot column = largest |.| among unused
columns (stop if |pivot| < 1e-15); residual column / pivot -> u, row -> v;
Frobenius estimate += |u|^2 |v|^2 + 2 Re sum_l (U_l^H u)(V_l^H v); stop when
|u||v| < htol sqrt(estimate); next row = largest |u| among unused rows.
Returns U (m x r), V (n x r) with A ~ U V^T.
"""
import numpy as np


def aca_block(A, htol=1e-6, kmax=100):
    m, n = A.shape
    kc = min(m, n, kmax)
    U = np.zeros((m, kc), dtype=complex)
    V = np.zeros((n, kc), dtype=complex)
    used_r = np.zeros(m, dtype=bool)
    used_c = np.zeros(n, dtype=bool)
    p = 0
    frob = 0.0
    r = 0
    for k in range(kc):
        row = A[p, :] - V[:, :r] @ U[p, :r]
        ar = np.abs(row)
        ar[used_c] = 0.0
        pc = int(np.argmax(ar))
        pv = row[pc]
        if abs(pv) < 1e-15:
            break
        col = A[:, pc] - U[:, :r] @ V[pc, :r]
        u = col / pv
        v = row.copy()
        U[:, r] = u
        V[:, r] = v
        r += 1
        used_r[p] = True
        used_c[pc] = True
        new_sq = np.vdot(u, u).real * np.vdot(v, v).real
        cross = 0.0
        if r > 1:
            cross = 2.0 * float(np.real(np.dot(np.conj(U[:, :r - 1].T) @ u, np.conj(V[:, :r - 1].T) @ v)))
        frob += new_sq + cross
        if frob > 0 and np.sqrt(new_sq) < htol * np.sqrt(abs(frob)):
            break
        au = np.abs(u)
        au[used_r] = 0.0
        p = int(np.argmax(au))
    return U[:, :r], V[:, :r]


def hmatrix_full(tree, dense, lowrank, A, htol=1e-6, kmax=100):
    """Dense reconstruction (particle order) of the H-matrix of A: dense
    blocks exact, admissible blocks by aca_block.  Also returns the ranks."""
    c2p = tree.ind[:, 0]
    Ac = A[np.ix_(c2p, c2p)]
    out = np.zeros_like(Ac)
    ranks = []
    for i1, i2 in dense:
        r0, r1 = tree.cind[i1]
        c0, c1 = tree.cind[i2]
        out[r0:r1 + 1, c0:c1 + 1] = Ac[r0:r1 + 1, c0:c1 + 1]
    for i1, i2 in lowrank:
        r0, r1 = tree.cind[i1]
        c0, c1 = tree.cind[i2]
        U, V = aca_block(Ac[r0:r1 + 1, c0:c1 + 1], htol, kmax)
        ranks.append(U.shape[1])
        out[r0:r1 + 1, c0:c1 + 1] = U @ V.T
    p2c = tree.ind[:, 1]
    return out[np.ix_(p2c, p2c)], np.array(ranks)
