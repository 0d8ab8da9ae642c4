"""Oracle: retarded Green function with near-field refinement (numpy, complex128).

Test infrastructure only (see ``oracle/__init__.py``).  Inputs are particles
built by ``mnpbem_b200.geometry`` (pinned against the reference meshes by
``tests/test_geometry.py``); outputs are the refinement coefficients and the
dense Green matrices of the reference ``CompGreenRet``.
"""
import math

import numpy as np

EPS = np.finfo(float).eps


# --------------------------------------------------------------------------- a1
def refinematrix(pos1, pos2, rad1, rad2, abs_cutoff=0.0, rel_cutoff=3.0):
    """Classify element pairs: 2 = coincident centroids, 1 = near, 0 = far.

    Reference: mnpbem/greenfun/refine_utils.py:29-158 with the algebraic
    distance of refine_utils.py:12-26 (d^2 = |p1|^2 + |p2|^2 - 2 p1.p2,
    d^2 < 1e-10 -> 0).  Returns (row, col, kind) in row-major order.
    """
    n1sq = np.sum(pos1 * pos1, axis=1)
    n2sq = np.sum(pos2 * pos2, axis=1)
    dsq = n1sq[:, None] + n2sq[None, :] - 2.0 * (pos1 @ pos2.T)
    dsq[dsq < 1e-10] = 0.0
    d = np.sqrt(dsq)
    d2 = d - rad2[None, :]
    idrel = d2 / rad1[:, None]
    kind = np.zeros(d.shape, dtype=np.int8)
    kind[((d2 < abs_cutoff) | (idrel < rel_cutoff)) & (d != 0)] = 1
    kind[d == 0] = 2
    row, col = np.nonzero(kind)
    return row, col, kind[row, col].astype(np.int32)


# --------------------------------------------------------------------------- a2
def refine_diag(p1, p2, rows, cols, order=5):
    """Self-element integrals by polar quadrature (cart derivative).

    g_n = sum_q w r^(n-1) / n!;  f = n f1 + t1 f2 + t2 f3 with
    f1_n = sum w (n-1)(n.r) r^(n-3)/n!, f{2,3}_n = sum w (n-1)(t.r) r^n / rr^3 / n!,
    rr = max(r, 1e-4 max r).
    Reference: mnpbem/greenfun/greenret_refined.py:122-285 (MATLAB
    Greenfun/@greenret/private/init.m:44-95).
    """
    nd = len(rows)
    g = np.zeros((nd, order + 1))
    f = np.zeros((nd, 3, order + 1))
    if nd == 0:
        return g, f
    pos, w, row = p2.quadpol(cols)
    counts = np.bincount(row, minlength=nd)
    npts = int(counts[0])
    if np.any(counts != npts):
        # mixed triangle / quad faces: integrate face by face
        for k in range(nd):
            sel = row == k
            gk, fk = _diag_integrals(p1, rows[k:k + 1], pos[sel][None], w[sel][None], order)
            g[k], f[k] = gk[0], fk[0]
        return g, f
    return _diag_integrals(p1, rows, pos.reshape(nd, npts, 3), w.reshape(nd, npts), order)


def _diag_integrals(p1, rows, pts, w, order):
    pos1 = p1.pos[rows]
    nv = p1.nvec[rows]
    t1 = p1.tvec1[rows]
    t2 = p1.tvec2[rows]
    vec = pos1[:, None, :] - pts
    r = np.maximum(np.sqrt(np.sum(vec * vec, axis=2)), EPS)
    ndr = np.einsum("ij,ikj->ik", nv, vec)
    in1 = np.einsum("ij,ikj->ik", t1, vec)
    in2 = np.einsum("ij,ikj->ik", t2, vec)
    rr = np.maximum(r, 1e-4 * r.max(axis=1, keepdims=True))
    g = np.zeros((len(rows), order + 1))
    f = np.zeros((len(rows), 3, order + 1))
    for n in range(order + 1):
        fac = math.factorial(n)
        g[:, n] = np.sum(w * r ** (n - 1), axis=1) / fac
        f1 = np.sum(w * (n - 1) * ndr * r ** (n - 3), axis=1) / fac
        f2 = np.sum(w * (n - 1) * in1 * r ** n / rr ** 3, axis=1) / fac
        f3 = np.sum(w * (n - 1) * in2 * r ** n / rr ** 3, axis=1) / fac
        f[:, :, n] = nv * f1[:, None] + t1 * f2[:, None] + t2 * f3[:, None]
    return g, f


# --------------------------------------------------------------------------- a3
def refine_offdiag(p1, p2, rows, cols, order=5):
    """Near-element integrals with the 28-point rule on (curved) sub-triangles.

    g_n = sum w (r - r0)^n / (r n!);  f_0 = -sum w (x,y,z)/r^3;
    f_n = sum w (x,y,z) [-(r-r0)^n/(r^3 n!) + (r-r0)^(n-1)/(r^2 (n-1)!)],
    r0 = |pos2_j - pos1_i|.
    Reference: mnpbem/greenfun/greenret_refined.py:287-516 (MATLAB init.m:98-177).
    """
    nr = len(rows)
    g = np.zeros((nr, order + 1))
    f = np.zeros((nr, 3, order + 1))
    if nr == 0:
        return g, f
    uface, inv = np.unique(cols, return_inverse=True)
    pos, wsp, row = p2.quad_integration(uface)
    wsp = wsp.tocsr()
    for k, face in enumerate(uface):
        sel = np.flatnonzero(inv == k)
        lo, hi = wsp.indptr[k], wsp.indptr[k + 1]
        idx = wsp.indices[lo:hi]
        wk = wsp.data[lo:hi]
        keep = wk > 0
        idx, wk = idx[keep], wk[keep]
        pts = pos[idx]
        src = p1.pos[rows[sel]]
        rv = src[:, None, :] - pts[None, :, :]
        r = np.maximum(np.sqrt(np.sum(rv * rv, axis=2)), EPS)
        v0 = p2.pos[face] - src
        r0 = np.sqrt(np.sum(v0 * v0, axis=1))
        dl = r - r0[:, None]
        for n in range(order + 1):
            g[sel, n] = (dl ** n / r / math.factorial(n)) @ wk
        fs = -1.0 / r ** 3
        for c in range(3):
            f[sel, c, 0] = (rv[..., c] * fs) @ wk
        for n in range(1, order + 1):
            fs = -dl ** n / (r ** 3 * math.factorial(n)) + dl ** (n - 1) / (r ** 2 * math.factorial(n - 1))
            for c in range(3):
                f[sel, c, n] = (rv[..., c] * fs) @ wk
    return g, f


# --------------------------------------------------------------------------- a4
def stat_F(cp, abs_cutoff=0.0, rel_cutoff=3.0):
    """Quasistatic surface derivative F_ij = -n_i.(r_i - r_j)/d^3 area_j of the
    compound particle with the quasistatic refinement (polar self terms, 28-point
    near terms).  Reference: mnpbem/greenfun/compgreen_stat.py:219-450."""
    pc = cp.pc
    pos, nvec, area = pc.pos, pc.nvec, pc.area
    r = pos[:, None, :] - pos[None, :, :]
    d = np.maximum(np.sqrt(np.sum(r * r, axis=2)), EPS)
    F = -np.sum(nvec[:, None, :] * r, axis=2) / d ** 3 * area[None, :]
    np.fill_diagonal(F, 0.0)
    rad = cp.bradius()
    rows, cols, kind = refinematrix(pos, pos, rad, rad, abs_cutoff, rel_cutoff)
    dsel = kind == 2
    if np.any(dsel):
        dr, dc = rows[dsel], cols[dsel]
        pq, wq, rq = pc.quadpol(dc)
        vec = pos[dr[rq]] - pq
        rr = np.maximum(np.linalg.norm(vec, axis=1), EPS)
        ndv = np.sum(vec * nvec[dr[rq]], axis=1)
        F[dr, dc] = -np.bincount(rq, weights=wq * ndv / rr ** 3, minlength=len(dr))[:len(dr)]
    nsel = kind == 1
    if np.any(nsel):
        nrow, ncol = rows[nsel], cols[nsel]
        uface = np.unique(ncol)
        pq, wsp, _ = pc.quad_integration(uface)
        wsp = wsp.tocsr()
        for k, face in enumerate(uface):
            nb = nrow[ncol == face]
            lo, hi = wsp.indptr[k], wsp.indptr[k + 1]
            idx, wk = wsp.indices[lo:hi], wsp.data[lo:hi]
            keep = wk > 0
            idx, wk = idx[keep], wk[keep]
            vec = pos[nb, None, :] - pq[idx][None, :, :]
            rr = np.maximum(np.linalg.norm(vec, axis=2), EPS)
            ndv = np.sum(nvec[nb, None, :] * vec, axis=2)
            F[nb, face] = -(ndv / rr ** 3) @ wk
    return F


def closed_corrections(cp, Fstat=None):
    """Per-particle diagonal corrections c_j = -2 pi dir - sum_i area_i F_ij / area_j
    over the faces i of the closed surface of particle j.

    Reference: mnpbem/greenfun/compgreen_ret.py:192-272 (initclosed) and
    :376-400 (the correction enters f[jj, :, 0] += c_j n_j).  Returns a list
    (one entry per particle) of arrays or None.
    """
    if Fstat is None:
        Fstat = stat_F(cp)
    area = cp.pc.area
    off = cp.offsets
    out = []
    for i, closed in enumerate(cp.closed_particles()):
        if closed is None:
            out.append(None)
            continue
        loc = np.concatenate([np.arange(off[c], off[c + 1]) for c in closed])
        ind = np.arange(off[i], off[i + 1])
        fsum = np.sum(area[loc][:, None] * Fstat[np.ix_(loc, ind)] / area[ind][None, :], axis=0)
        out.append(-2 * np.pi * 1.0 - fsum)
    return out


# --------------------------------------------------------------------------- a5
def connect(inout):
    """con[i][j][a, b] = material index connecting region i of particle a with
    region j of particle b, or 0 (reference compgreen_ret.py:435-505)."""
    io = np.asarray(inout)
    con = [[None, None], [None, None]]
    for i in range(2):
        for j in range(2):
            c1 = io[:, i][:, None]
            c2 = io[:, j][None, :]
            con[i][j] = np.where(c1 == c2, np.broadcast_to(c1, (len(io), len(io))), 0)
    return con


class RefinedBlock:
    """Refinement data of one particle pair (rows/cols local to the block)."""

    def __init__(self, rows, cols, kind, g, f):
        self.rows, self.cols, self.kind, self.g, self.f = rows, cols, kind, g, f


def refine_pair(pa, pb, order=5, abs_cutoff=0.0, rel_cutoff=3.0):
    """Refinement of the (pa, pb) particle block: GreenRetRefined.__init__
    (reference greenret_refined.py:49-120)."""
    rows, cols, kind = refinematrix(pa.pos, pb.pos, pa.bradius(), pb.bradius(), abs_cutoff, rel_cutoff)
    g = np.zeros((len(rows), order + 1))
    f = np.zeros((len(rows), 3, order + 1))
    d = kind == 2
    gd, fd = refine_diag(pa, pb, rows[d], cols[d], order)
    g[d], f[d] = gd, fd
    o = kind == 1
    go, fo = refine_offdiag(pa, pb, rows[o], cols[o], order)
    g[o], f[o] = go, fo
    return RefinedBlock(rows, cols, kind, g, f)


def refine_all(cp, order=5):
    """All particle-pair refinements plus the closed-surface correction
    (CompGreenRet._init, reference compgreen_ret.py:113-166)."""
    blocks = [[refine_pair(pa, pb, order) for pb in cp.p] for pa in cp.p]
    corr = closed_corrections(cp)
    for i, c in enumerate(corr):
        if c is None:
            continue
        blk = blocks[i][i]
        nv = cp.p[i].nvec
        dg = np.flatnonzero(blk.rows == blk.cols)
        blk.f[dg, :, 0] += c[blk.rows[dg]][:, None] * nv[blk.rows[dg]]
    return blocks


# --------------------------------------------------------------------------- a6
def green_block(pa, pb, blk, k, key, same):
    """G or F (cart derivative projected on n) of one particle block at complex
    wavenumber k: far field from centroids, refined entries overwritten by
    sum_n c_n (ik)^n, then multiplied by exp(ikd).  Keys Gp, H1p, H2p give the
    Cartesian derivative as an (na, 3, nb) array.
    Reference: mnpbem/greenfun/greenret_refined.py:654-864 (MATLAB eval1.m:18-153).
    """
    x = pa.pos[:, 0:1] - pb.pos[:, 0]
    y = pa.pos[:, 1:2] - pb.pos[:, 1]
    z = pa.pos[:, 2:3] - pb.pos[:, 2]
    d = np.maximum(np.sqrt(x ** 2 + y ** 2 + z ** 2), EPS)
    if same:
        np.fill_diagonal(d, EPS)
    ikp = np.array([(1j * k) ** n for n in range(blk.g.shape[1])])
    if key in ("Gp", "H1p", "H2p"):
        aux = (1j * k - 1.0 / d) / d ** 2 * pb.area[None, :]
        comps = []
        for c, r in enumerate((x, y, z)):
            M = aux * r + 0j
            M[blk.rows, blk.cols] = blk.f[:, c, :] @ ikp
            comps.append(M * np.exp(1j * k * d))
        Gp = np.stack(comps, axis=1)
        if same and key != "Gp":
            idx = np.arange(pa.n)
            Gp[idx, :, idx] += (2 * np.pi if key == "H1p" else -2 * np.pi) * pa.nvec
        return Gp
    if key == "G":
        M = (1.0 / d) * pb.area[None, :] + 0j
        M[blk.rows, blk.cols] = blk.g @ ikp
    else:
        nv = pa.nvec
        aux = (1j * k - 1.0 / d) / d ** 2
        M = (nv[:, 0:1] * (aux * x) + nv[:, 1:2] * (aux * y) + nv[:, 2:3] * (aux * z)) * pb.area[None, :]
        M[blk.rows, blk.cols] = np.einsum("ij,ijk,k->i", nv[blk.rows], blk.f, ikp)
    M = M * np.exp(1j * k * d)
    if key == "H1" and same:
        M[np.diag_indices_from(M)] += 2 * np.pi
    if key == "H2" and same:
        M[np.diag_indices_from(M)] -= 2 * np.pi
    return M


def green_region(cp, blocks, i, j, key, enei):
    """CompGreenRet._eval1 for region pair (i, j) (reference compgreen_ret.py:739-858).
    Returns the dense (N, N) matrix or the int 0 when nothing connects."""
    con = connect(cp.inout)[i][j]
    ks = [m(enei)[1] for m in cp.eps]
    off = cp.offsets
    M = None
    cart = key in ("Gp", "H1p", "H2p")
    for a in range(len(cp.p)):
        for b in range(len(cp.p)):
            if con[a, b] > 0:
                if M is None:
                    M = np.zeros((cp.n, 3, cp.n) if cart else (cp.n, cp.n), dtype=complex)
                kb = complex(np.asarray(ks[con[a, b] - 1]).ravel()[0])
                M[off[a]:off[a + 1], ..., off[b]:off[b + 1]] = green_block(
                    cp.p[a], cp.p[b], blocks[a][b], kb, key, a == b)
    if M is None or np.all(M == 0):
        return 0
    return M


def bem_matrices(cp, blocks, enei):
    """G1 = G11 - G21, G2 = G22 - G12, H1 = H1_11 - H1_21, H2 = H2_22 - H2_12
    (reference mnpbem/bem/bem_ret.py:407-423)."""
    def sub(a, b):
        if isinstance(b, int):
            return a
        if isinstance(a, int):
            return -b
        return a - b
    G1 = sub(green_region(cp, blocks, 0, 0, "G", enei), green_region(cp, blocks, 1, 0, "G", enei))
    G2 = sub(green_region(cp, blocks, 1, 1, "G", enei), green_region(cp, blocks, 0, 1, "G", enei))
    H1 = sub(green_region(cp, blocks, 0, 0, "H1", enei), green_region(cp, blocks, 1, 0, "H1", enei))
    H2 = sub(green_region(cp, blocks, 1, 1, "H2", enei), green_region(cp, blocks, 0, 1, "H2", enei))
    return G1, G2, H1, H2


# --------------------------------------------------------------------------- f4
def _mm(M, x):
    """Matrix (n, n) or derivative (n, 3, n) times a vector field over the
    last axis of M (reference CompGreenRet._matmul, compgreen_ret.py:1040-1098).
    The int 0 (no connected block) gives 0."""
    if isinstance(M, int):
        return 0
    return np.tensordot(M, x, axes=([M.ndim - 1], [0]))


def _cross(Gp, h):
    """Gp x h with Gp (n, 3, n) and h (n, 3, p) (reference CompGreenRet._cross,
    compgreen_ret.py:1100-1136)."""
    if isinstance(Gp, int):
        return 0
    out = np.zeros((Gp.shape[0], 3, h.shape[2]), dtype=complex)
    for c in range(3):
        c1, c2 = (c + 1) % 3, (c + 2) % 3
        out[:, c] = Gp[:, c1, :] @ h[:, c2, :] - Gp[:, c2, :] @ h[:, c1, :]
    return out


def potential(cp, blocks, sig1, sig2, h1, h2, enei, inout):
    """Potentials and surface derivatives of a solution inside (inout 1) or
    outside (inout 2): phi, phip (n, p), a, ap (n, 3, p).
    Reference: CompGreenRet.potential, mnpbem/greenfun/compgreen_ret.py:976-1038."""
    r = inout - 1
    hk = "H1" if inout == 1 else "H2"
    G1, G2 = green_region(cp, blocks, r, 0, "G", enei), green_region(cp, blocks, r, 1, "G", enei)
    H1, H2 = green_region(cp, blocks, r, 0, hk, enei), green_region(cp, blocks, r, 1, hk, enei)
    phi = _mm(G1, sig1) + _mm(G2, sig2)
    phip = _mm(H1, sig1) + _mm(H2, sig2)
    a = _mm(G1, h1) + _mm(G2, h2)
    ap = _mm(H1, h1) + _mm(H2, h2)
    return phi, phip, a, ap


def field(cp, blocks, sig1, sig2, h1, h2, enei, inout):
    """Electric and magnetic fields at the faces, inside (inout 1) or outside
    (inout 2): e, h (n, 3, p).
    Reference: CompGreenRet.field, mnpbem/greenfun/compgreen_ret.py:912-974."""
    r = inout - 1
    k = 2 * np.pi / enei
    hk = "H1p" if inout == 1 else "H2p"
    G1, G2 = green_region(cp, blocks, r, 0, "G", enei), green_region(cp, blocks, r, 1, "G", enei)
    e = 1j * k * (_mm(G1, h1) + _mm(G2, h2))
    P1, P2 = green_region(cp, blocks, r, 0, hk, enei), green_region(cp, blocks, r, 1, hk, enei)
    e = e - _mm(P1, sig1) - _mm(P2, sig2)
    h = _cross(P1, h1) + _cross(P2, h2)
    return e, h
