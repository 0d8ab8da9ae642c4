"""H-matrix (hierarchical low-rank) representation of the BEM matrices on the GPU.

Host side (geometry only, once per mesh / wavelength):

* ``ClusterTree``   -- recursive bisection of the face centroids with a first
  split per particle (reference mnpbem/greenfun/clustertree.py:7-380, after
  Boerm et al., Eng. Anal. Bound. Elem. 27, 405 (2003));
* ``block_partition`` -- admissibility recursion over cluster pairs: leaf x
  leaf pairs are dense blocks, admissible pairs low-rank blocks
  (clustertree.py:304-376), with the wavenumber-aware criterion of
  ``make_kaware_fadmiss`` (mnpbem/greenfun/hmatrix.py:1284-1310).

Device side (libbem200, csrc/hmat.cu):

* the dense BEM matrix is gathered into cluster order; low-rank blocks are
  compressed by partially pivoted adaptive cross approximation, one CTA per
  block, with the reference's pivoting and stopping rule
  (hmatrix.py:195-336, tolerance ``htol``, rank <= ``kmax``); dense leaves are
  packed;
* the product H x runs in two kernels: T_b = V_b^T x for every low-rank block,
  then one CTA per block adds its rows, M_b times the block's x (or T) slice,
  into y (reference HMatrix.mtimes_vec, hmatrix.py:450-541).

The reference compresses each region-pair Green matrix (G11, G21, ...) and
forms G1 = G11 - G21 by H-matrix addition with QR/SVD recompression
(hmatrix.py:580-737).  Here the combined BEM matrices G1, G2, H1, H2 are
assembled densely on the GPU and compressed directly, which approximates the
same operators to the same tolerance.
"""
import ctypes

import numpy as np

from . import _native as nat


def _torch():
    import torch
    return torch


# --------------------------------------------------------------------------- tree
class ClusterTree:
    """Cluster tree of face centroids (reference clustertree.py:7-146).

    Attributes (0-based): son (nnodes, 2) children or -1, cind (nnodes, 2)
    first/last cluster index, mid (nnodes, 3), rad (nnodes,), ipart (nnodes,)
    particle of the node or -1, ind (n, 2): ind[c, 0] = face of cluster index
    c, ind[f, 1] = cluster index of face f.
    """

    def __init__(self, pos, cleaf=32, ipart_arr=None):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.n = self.pos.shape[0]
        self._ipart = (np.zeros(self.n, dtype=np.int64) if ipart_arr is None
                       else np.asarray(ipart_arr, dtype=np.int64))
        self._build(int(cleaf))

    def _sphere(self, ind):
        p = self.pos[ind]
        lo, hi = p.min(axis=0), p.max(axis=0)
        return 0.5 * (lo + hi), 0.5 * float(np.linalg.norm(hi - lo))

    def _split(self, ind):
        ip = self._ipart[ind]
        if np.any(ip != ip[0]):  # first split: first particle against the rest
            mask = ip == ip[0]
            return ind[mask], ind[~mask], True
        p = self.pos[ind]
        lo, hi = p.min(axis=0), p.max(axis=0)
        ext = hi - lo
        k = int(np.argmax(ext))
        mask = self.pos[ind, k] < lo[k] + 0.5 * ext[k]
        i1, i2 = ind[mask], ind[~mask]
        if len(i1) == 0:
            i1, i2 = ind[:1], ind[1:]
        elif len(i2) == 0:
            i1, i2 = ind[:-1], ind[-1:]
        return i1, i2, False

    def _build(self, cleaf):
        n = self.n
        lo, hi = self.pos.min(axis=0), self.pos.max(axis=0)
        nodes = [dict(cs=0, ce=n - 1, mid=0.5 * (lo + hi), rad=0.5 * float(np.linalg.norm(hi - lo)), s1=-1, s2=-1,
                      leaf=None)]
        # explicit stack in the reference's recursion order (son 1 subtree, then son 2)
        stack = [(0, np.arange(n, dtype=np.int64), np.arange(n, dtype=np.int64))]
        while stack:
            ic, ind, cind = stack.pop()
            base = len(nodes)
            nodes[ic]["s1"], nodes[ic]["s2"] = base, base + 1
            i1, i2, psplit = self._split(ind)
            c1, c2 = cind[:len(i1)], cind[len(i1):]
            for ii, cc in ((i1, c1), (i2, c2)):
                m, r = self._sphere(ii)
                nodes.append(dict(cs=int(cc[0]), ce=int(cc[-1]), mid=m, rad=r, s1=-1, s2=-1, leaf=None))
            todo = []
            for off, ii, cc in ((0, i1, c1), (1, i2, c2)):
                if len(ii) > cleaf or psplit:
                    todo.append((base + off, ii, cc))
                else:
                    nodes[base + off]["leaf"] = ii
            stack.extend(reversed(todo))  # son 1 is expanded first
        nn = len(nodes)
        self.son = np.array([[d["s1"], d["s2"]] for d in nodes], dtype=np.int64)
        self.cind = np.array([[d["cs"], d["ce"]] for d in nodes], dtype=np.int64)
        self.mid = np.array([d["mid"] for d in nodes], dtype=np.float64)
        self.rad = np.array([d["rad"] for d in nodes], dtype=np.float64)
        c2p = np.empty(n, dtype=np.int64)
        for d in nodes:
            if d["leaf"] is not None:
                c2p[d["cs"]:d["ce"] + 1] = d["leaf"]
        p2c = np.empty(n, dtype=np.int64)
        p2c[c2p] = np.arange(n)
        self.ind = np.stack([c2p, p2c], axis=1)
        ip = np.empty(nn, dtype=np.int64)
        for i, d in enumerate(nodes):
            a, b = self._ipart[c2p[d["cs"]]], self._ipart[c2p[d["ce"]]]
            ip[i] = a if a == b else -1
        self.ipart = ip

    def is_leaf(self, i):
        return self.son[i, 0] == -1


def eta_fadmiss(eta=2.5):
    """Boerm's criterion eta * min(rad1, rad2) < dist (clustertree.py:311)."""
    return lambda r1, r2, d: eta * min(r1, r2) < d


def make_kaware_fadmiss(k, eta0=2.5):
    """Wavenumber-aware admissibility (reference hmatrix.py:1284-1310): the
    Boerm criterion, and for clusters wider than 1/|k| also a distance of at
    least one wavelength."""
    if k is None or not np.isfinite(k) or abs(k) < 1e-12:
        return eta_fadmiss(eta0)
    ka = abs(complex(k))
    lam = 2.0 * np.pi / ka

    def fadmiss(r1, r2, d):
        rmin = min(r1, r2)
        if eta0 * rmin >= d:
            return False
        if ka * rmin > 1.0 and d < lam:
            return False
        return True
    return fadmiss


def block_partition(tree, fadmiss):
    """Dense (leaf x leaf) and low-rank (admissible) cluster pairs, in the
    reference's recursion order (clustertree.py:324-376)."""
    dense, lowrank = [], []

    def admissible(i1, i2):
        if tree.is_leaf(i1) and tree.is_leaf(i2):
            return 2
        if tree.ipart[i1] == -1 or tree.ipart[i2] == -1:
            return 0
        d = float(np.linalg.norm(tree.mid[i1] - tree.mid[i2]))
        return 1 if fadmiss(tree.rad[i1], tree.rad[i2], d) else 0

    stack = [(0, 0)]
    while stack:
        i1, i2 = stack.pop()
        ad = admissible(i1, i2)
        if ad == 2:
            dense.append((i1, i2))
        elif ad == 1:
            lowrank.append((i1, i2))
        else:
            s1 = [i1] if tree.is_leaf(i1) else [tree.son[i1, 0], tree.son[i1, 1]]
            s2 = [i2] if tree.is_leaf(i2) else [tree.son[i2, 0], tree.son[i2, 1]]
            stack.extend(reversed([(a, b) for a in s1 for b in s2]))
    return dense, lowrank


# --------------------------------------------------------------------------- device H-matrix
class HMatrixGPU:
    """Compressed n x n complex128 matrix on the device (cluster order).

    ``compress(M)`` takes the dense matrix in particle order; ``matvec(x, y)``
    computes y = H x for n x w row-major device arrays in cluster order.
    """

    def __init__(self, tree, dense, lowrank, htol=1e-6, kmax=100, device="cuda"):
        torch = _torch()
        self.tree = tree
        self.n = tree.n
        self.htol = float(htol)
        self.kmax = int(kmax)
        dev = torch.device(device)
        self.dev = dev
        cind = tree.cind

        def rng(i):
            return int(cind[i, 0]), int(cind[i, 1] - cind[i, 0] + 1)

        # dense leaves: (r0, m, c0, nb) and packed offsets
        db = np.array([[*rng(a), *rng(b)] for a, b in dense], dtype=np.int32).reshape(-1, 4)
        doff = np.zeros(len(db) + 1, dtype=np.int64)
        doff[1:] = np.cumsum(db[:, 1].astype(np.int64) * db[:, 3])
        # low-rank blocks, storage for the maximum rank min(m, nb, kmax)
        lb = np.array([[*rng(a), *rng(b)] for a, b in lowrank], dtype=np.int32).reshape(-1, 4)
        kcap = np.minimum(np.minimum(lb[:, 1], lb[:, 3]), self.kmax).astype(np.int64)
        uoff = np.zeros(len(lb) + 1, dtype=np.int64)
        uoff[1:] = np.cumsum(lb[:, 1].astype(np.int64) * kcap)
        voff = np.zeros(len(lb) + 1, dtype=np.int64)
        voff[1:] = np.cumsum(lb[:, 3].astype(np.int64) * kcap)
        toff = np.zeros(len(lb) + 1, dtype=np.int64)
        toff[1:] = np.cumsum(kcap)
        self.ndense, self.nlow = len(db), len(lb)
        self._db, self._lb, self._kcap = db, lb, kcap
        self._doff_h, self._uoff_h, self._voff_h = doff, uoff, voff
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
        self.dblk, self.doff = t(db.reshape(-1)), t(doff)
        self.lblk, self.uoff, self.voff, self.toff = t(lb.reshape(-1)), t(uoff), t(voff), t(toff)
        self.kcap = t(kcap.astype(np.int32))
        self.D = torch.empty(max(int(doff[-1]), 1), dtype=torch.complex128, device=dev)
        self.U = torch.empty(max(int(uoff[-1]), 1), dtype=torch.complex128, device=dev)
        self.V = torch.empty(max(int(voff[-1]), 1), dtype=torch.complex128, device=dev)
        self.rank = torch.zeros(max(len(lb), 1), dtype=torch.int32, device=dev)
        self.c2p = t(tree.ind[:, 0].astype(np.int32))
        self.p2c = t(tree.ind[:, 1].astype(np.int32))
        self.ranks = None
        # work items of the product: (low-rank block, first V row) per 128 rows
        # of V, and (block, first row) per 32 rows of every block (dense first)
        vit = [(l, j0) for l in range(len(lb)) for j0 in range(0, int(lb[l, 3]), 128)]
        bit = [(b, i0) for b in range(len(db)) for i0 in range(0, int(db[b, 1]), 32)]
        bit += [(len(db) + l, i0) for l in range(len(lb)) for i0 in range(0, int(lb[l, 1]), 32)]
        self.nvitems, self.nbitems = len(vit), len(bit)
        self.vitems = t(np.array(vit, dtype=np.int32).reshape(-1))
        self.bitems = t(np.array(bit, dtype=np.int32).reshape(-1))

    def compress(self, M, scratch=None):
        """Compress the dense n x n complex128 device matrix M (particle order)."""
        torch = _torch()
        n = self.n
        Mc = scratch if scratch is not None else torch.empty((n, n), dtype=torch.complex128, device=self.dev)
        s = nat.stream_ptr()
        nat.call("bem200_hmat_permute", n, nat.ptr(M), nat.ptr(self.c2p), nat.ptr(Mc), s)
        if self.ndense:
            nat.call("bem200_hmat_pack_dense", self.ndense, nat.ptr(self.dblk), nat.ptr(self.doff), n, nat.ptr(Mc),
                     nat.ptr(self.D), s)
        if self.nlow:
            max_rows = int(max(self._lb[:, 1].max(), self._lb[:, 3].max()))
            nat.call("bem200_hmat_aca", self.nlow, nat.ptr(self.lblk), nat.ptr(self.uoff), nat.ptr(self.voff),
                     nat.ptr(self.kcap), n, nat.ptr(Mc), self.htol, nat.ptr(self.U), nat.ptr(self.V),
                     nat.ptr(self.rank), max_rows, int(self._kcap.max()), s)
            self.ranks = self.rank.cpu().numpy()[:self.nlow].copy()
        else:
            self.ranks = np.zeros(0, dtype=np.int32)
        return self

    def compress_green(self, g, enei, which):
        """Compress BEM matrix ``which`` (0 = G1, 1 = G2, 2 = H1, 3 = H2) of the
        Green function ``g`` (a CompGreenRet) at ``enei`` with every entry of the
        dense leaves and of the ACA rows and columns computed on demand: no
        n x n matrix is formed (bem200_hmat_compress_green)."""
        ks = g.wavenumbers(enei)
        kmat = (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])
        blk = g._blk_mat([(0, 0), (1, 0), (1, 1), (0, 1)])
        r = g.refined
        has_ref = r.nref > 0
        max_rows = int(max(self._lb[:, 1].max(), self._lb[:, 3].max())) if self.nlow else 1
        max_kcap = int(self._kcap.max()) if self.nlow else 1
        nat.call("bem200_hmat_compress_green", int(which), self.n, g.npart, nat.ptr(g.pid), nat.ptr(blk), len(ks),
                 ctypes.cast(kmat, ctypes.c_void_p), nat.ptr(g.pos), nat.ptr(g.nvec), nat.ptr(g.area),
                 nat.ptr(r.row_ptr) if has_ref else None, nat.ptr(r.col) if has_ref else None, g.order,
                 nat.ptr(r.g) if has_ref else None, nat.ptr(r.fn) if has_ref else None, nat.ptr(self.c2p),
                 self.ndense, nat.ptr(self.dblk), nat.ptr(self.doff), nat.ptr(self.D), self.nlow, nat.ptr(self.lblk),
                 nat.ptr(self.uoff), nat.ptr(self.voff), nat.ptr(self.kcap), self.htol, nat.ptr(self.U),
                 nat.ptr(self.V), nat.ptr(self.rank), max_rows, max_kcap, nat.stream_ptr())
        self.ranks = self.rank.cpu().numpy()[:self.nlow].copy() if self.nlow else np.zeros(0, dtype=np.int32)
        return self

    def compression(self):
        """Stored elements / n^2 (reference HMatrix.compression, hmatrix.py:739-756)."""
        ne = int(self._doff_h[-1]) + int(np.sum(self.ranks.astype(np.int64) * (self._lb[:, 1] + self._lb[:, 3])))
        return ne / float(self.n * self.n)

    def matvec(self, x, y, w):
        """y = H x, x and y n x w row-major complex128 in cluster order, with
        large blocks split over several CTAs (bem200_hmat_matvec_items)."""
        torch = _torch()
        tbuf = getattr(self, "_tbuf", None)
        need = max(int(np.sum(self._kcap)) * w, 1)
        if tbuf is None or tbuf.numel() < need:
            self._tbuf = tbuf = torch.empty(need, dtype=torch.complex128, device=self.dev)
        nat.call("bem200_hmat_matvec_items", self.n, w, nat.ptr(x), self.nlow, nat.ptr(self.lblk),
                 nat.ptr(self.voff), nat.ptr(self.uoff), nat.ptr(self.toff), nat.ptr(self.kcap), nat.ptr(self.rank),
                 nat.ptr(self.U), nat.ptr(self.V), nat.ptr(tbuf), int(np.sum(self._kcap)) * w, self.ndense,
                 nat.ptr(self.dblk), nat.ptr(self.doff), nat.ptr(self.D), self.nvitems, nat.ptr(self.vitems),
                 self.nbitems, nat.ptr(self.bitems), nat.ptr(y), nat.stream_ptr())

    def matvec_per_block(self, x, y, w):
        """y = H x with one CTA per block (bem200_hmat_matvec)."""
        torch = _torch()
        tbuf = getattr(self, "_tbuf", None)
        need = max(int(np.sum(self._kcap)) * w, 1)
        if tbuf is None or tbuf.numel() < need:
            self._tbuf = tbuf = torch.empty(need, dtype=torch.complex128, device=self.dev)
        nat.call("bem200_hmat_matvec", self.n, w, nat.ptr(x), self.nlow, nat.ptr(self.lblk), nat.ptr(self.voff),
                 nat.ptr(self.uoff), nat.ptr(self.toff), nat.ptr(self.kcap), nat.ptr(self.rank), nat.ptr(self.U),
                 nat.ptr(self.V), nat.ptr(tbuf), self.ndense, nat.ptr(self.dblk), nat.ptr(self.doff),
                 nat.ptr(self.D), nat.ptr(y), nat.stream_ptr())


def particle_index(p):
    """Particle of every face of a compound particle (or None for one particle)."""
    if not hasattr(p, "p") or len(p.p) <= 1:
        return None
    off = np.asarray(p.offsets)
    return np.repeat(np.arange(len(p.p)), np.diff(off)).astype(np.int64)


class BEMHMatrices:
    """G1, G2, H1, H2 of the BEM as device H-matrices and the BEM operator on them.

    ``build(enei)`` compresses the four matrices (wavenumber-aware
    admissibility at k = 2 pi / enei, as the reference ACACompGreenRet.eval,
    aca_compgreen_ret.py:156-164): from dense matrices already at hand, or
    with entries computed on demand from the Green function (the default when
    none are given); ``apply`` is the FP64 operator of ``bem200_bem_apply``
    with the four products done by H-matrix matvecs.
    """

    def __init__(self, p, g, htol=1e-6, kmax=(4, 100), cleaf=200, eta=2.5):
        self.p = p
        self.g = g
        self.n = p.n
        self.htol = float(max(htol) if hasattr(htol, "__iter__") else htol)
        self.kmax = int(max(kmax) if hasattr(kmax, "__iter__") else kmax)
        self.cleaf = int(cleaf)
        self.eta = float(eta)
        self.tree = ClusterTree(p.pos, cleaf=self.cleaf, ipart_arr=particle_index(p))
        self.H = None
        self.enei = None

    def build(self, enei, mats=None, fill="green"):
        """Compress G1, G2, H1, H2 at ``enei``.  ``mats`` may hand in the four
        dense complex128 matrices already assembled at this wavelength;
        without them, fill='green' computes every stored entry on demand from
        the Green function (no n x n matrix), fill='dense' assembles the dense
        matrices first."""
        torch = _torch()
        n = self.n
        fad = make_kaware_fadmiss(2.0 * np.pi / enei, eta0=self.eta)
        dense, low = block_partition(self.tree, fad)
        dev = self.g.device
        if mats is None and fill == "green":
            self.H = None
            self.H = [HMatrixGPU(self.tree, dense, low, htol=self.htol, kmax=self.kmax).compress_green(self.g, enei, w)
                      for w in range(4)]
            self.enei = enei
            return self
        if fill not in ("green", "dense"):
            raise ValueError("BEMHMatrices.build: fill must be 'green' or 'dense'")
        if mats is None:
            mats = [torch.empty((n, n), dtype=torch.complex128, device=dev) for _ in range(4)]
            self.g.bem_matrices(enei, dtype="c128", out=mats)
        self.H = None
        scratch = torch.empty((n, n), dtype=torch.complex128, device=dev)
        self.H = [HMatrixGPU(self.tree, dense, low, htol=self.htol, kmax=self.kmax).compress(M, scratch) for M in mats]
        del mats, scratch
        self.enei = enei
        return self

    def compression(self):
        return [h.compression() for h in self.H]

    def apply(self, npol, eps_mode, e1p, e2p, nvec, k0, x, out):
        """out = A x (the full BEM operator) for x in the solution layout."""
        torch = _torch()
        n = self.n
        w = 8 * npol
        np_ = n * npol
        dev = x.device
        key = npol
        if getattr(self, "_bufkey", None) != key:
            self._U = [torch.empty((n, w), dtype=torch.complex128, device=dev) for _ in range(2)]
            self._Uc = [torch.empty((n, w), dtype=torch.complex128, device=dev) for _ in range(2)]
            self._Yc = torch.empty((n, w), dtype=torch.complex128, device=dev)
            self._Y = [torch.empty((n, w), dtype=torch.complex128, device=dev) for _ in range(4)]
            self._bufkey = key
        s = nat.stream_ptr()
        base = x.data_ptr()
        c2p, p2c = self.H[0].c2p, self.H[0].p2c
        for side in range(2):
            nat.call("bem200_op_prep", n, npol, ctypes.c_void_p(base + 16 * 4 * np_ * side), eps_mode, e1p, e2p,
                     side, nat.ptr(self._U[side]), s)
            nat.call("bem200_hmat_gather_rows", n, w, nat.ptr(self._U[side]), nat.ptr(c2p), nat.ptr(self._Uc[side]), s)
        # G1 U1, G2 U2, H1 U1, H2 U2 in cluster order, back to particle order
        for i, (h, side) in enumerate(zip(self.H, (0, 1, 0, 1))):
            h.matvec(self._Uc[side], self._Yc, w)
            nat.call("bem200_hmat_gather_rows", n, w, nat.ptr(self._Yc), nat.ptr(p2c), nat.ptr(self._Y[i]), s)
        nat.call("bem200_op_combine", n, npol, nat.ptr(self._Y[0]), nat.ptr(self._Y[1]), nat.ptr(self._Y[2]),
                 nat.ptr(self._Y[3]), nat.ptr(nvec), k0, None, nat.ptr(out), s)
