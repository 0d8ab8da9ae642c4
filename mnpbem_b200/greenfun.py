"""Retarded Green function of a compound particle, evaluated on the GPU.

``CompGreenRet(p, p)`` mirrors the reference class (mnpbem/greenfun/
compgreen_ret.py:14): construction computes the near-field refinement once
per mesh, ``eval(i, j, key, enei)`` returns one region-pair matrix and
``bem_matrices(enei)`` returns the four BEM matrices G1, G2, H1, H2 in one
fused kernel pass.  All work runs in libbem200 kernels:

* refinement classification (refinematrix)          -> bem200_refine_count/fill
* polar / 28-point refinement integrals             -> bem200_refine_integrals
* closed-surface (Fuchs-Liu) diagonal correction    -> bem200_closed_correction
* far field + refined overlay + e^{ikd}             -> bem200_green_assemble
* Cartesian derivatives Gp, H1p, H2p                -> bem200_green_assemble_cart
* potentials / fields of a solution at the faces    -> bem200_green_potential / _field
  (entries computed on the fly, no n x n matrix stored)
"""
import ctypes

import numpy as np

from . import _native as nat


def connect(inout):
    """Region connectivity con[i][j][a, b] (reference compgreen_ret.py:435-505)."""
    io = np.asarray(inout)
    con = [[None, None], [None, None]]
    for i in range(2):
        for j in range(2):
            c1 = io[:, i][:, None]
            c2 = io[:, j][None, :]
            con[i][j] = np.where(c1 == c2, np.broadcast_to(c1, (len(io), len(io))), 0).astype(np.int32)
    return con


def _torch():
    import torch
    return torch


class Refinement:
    """Device arrays of the refined entries: row, col, kind, g (nref, order+1),
    f (nref, 3, order+1), fn = n_row . f (nref, order+1)."""


class CompGreenRet:
    """Green function between the faces of a compound particle and itself.

    Options (reference defaults): order=5, RelCutoff=3, AbsCutoff=0,
    deriv='cart'.  Only ``p1 is p2`` (the BEM case) is supported.
    """

    def __init__(self, p1, p2=None, device="cuda", **options):
        torch = _torch()
        if p2 is not None and p2 is not p1:
            raise NotImplementedError("CompGreenRet: only the self interaction p1 is p2 is supported")
        if not torch.cuda.is_available():
            raise RuntimeError("CompGreenRet: a CUDA device is required (no CPU fallback)")
        self.p1 = self.p2 = p1
        self.order = int(options.get("order", 5))
        self.rel_cutoff = float(options.get("RelCutoff", 3))
        self.abs_cutoff = float(options.get("AbsCutoff", 0))
        self.deriv = options.get("deriv", "cart")
        if self.deriv != "cart":
            raise NotImplementedError("CompGreenRet: only deriv='cart' is supported")
        self.device = torch.device(device)
        self.con = connect(p1.inout)
        self.n = p1.n
        self._upload()
        self._refine()

    # ------------------------------------------------------------ inputs
    def _upload(self):
        torch = _torch()
        cp = self.p1
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.pos = torch.as_tensor(np.ascontiguousarray(cp.pos), **f64)
        self.nvec = torch.as_tensor(np.ascontiguousarray(cp.nvec), **f64)
        self.tvec1 = torch.as_tensor(np.ascontiguousarray(cp.tvec1), **f64)
        self.tvec2 = torch.as_tensor(np.ascontiguousarray(cp.tvec2), **f64)
        self.area = torch.as_tensor(np.ascontiguousarray(cp.area), **f64)
        self.rad = torch.as_tensor(np.ascontiguousarray(cp.bradius()), **f64)
        nodes, kinds = [], []
        for q in cp.p:
            nd, kd = q.node_table()
            nodes.append(nd)
            kinds.append(kd)
        self.nodes = torch.as_tensor(np.ascontiguousarray(np.concatenate(nodes)), **f64)
        self.face_kind = torch.as_tensor(np.concatenate(kinds).astype(np.int32), device=dev)
        q = cp.p[0].quad
        self.n28, self.n3, self.n4 = len(q.x), len(q.x3), len(q.x4)
        rules = np.concatenate([q.x, q.y, q.w, q.x3, q.y3, q.w3, q.x4, q.y4, q.w4])
        self.rules = torch.as_tensor(rules, **f64)
        off = cp.offsets
        npart = len(cp.p)
        self.npart = npart
        pid = np.repeat(np.arange(npart), np.diff(off)).astype(np.int32)
        self.pid = torch.as_tensor(pid, device=dev)
        mask = np.zeros(npart, dtype=np.uint64)
        for i, c in enumerate(cp.closed_particles()):
            if c is not None:
                for k in c:
                    mask[i] |= np.uint64(1) << np.uint64(k)
        self.closed_mask = torch.as_tensor(mask.view(np.int64), device=dev)

    # -------------------------------------------------------- refinement
    def _refine(self):
        torch = _torch()
        n = self.n
        dev = self.device
        s = nat.stream_ptr()
        counts = torch.empty(n, dtype=torch.int32, device=dev)
        nat.call("bem200_refine_count", n, nat.ptr(self.pos), nat.ptr(self.rad), self.abs_cutoff,
                 self.rel_cutoff, nat.ptr(counts), s)
        row_ptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
        nat.call("bem200_scan_i32", n, nat.ptr(counts), nat.ptr(row_ptr), s)
        nref = int(row_ptr[n].item())
        r = Refinement()
        r.nref = nref
        r.row_ptr = row_ptr
        r.row = torch.empty(max(nref, 1), dtype=torch.int32, device=dev)
        r.col = torch.empty(max(nref, 1), dtype=torch.int32, device=dev)
        r.kind = torch.empty(max(nref, 1), dtype=torch.int8, device=dev)
        nat.call("bem200_refine_fill", n, nat.ptr(self.pos), nat.ptr(self.rad), self.abs_cutoff, self.rel_cutoff,
                 nat.ptr(row_ptr), nat.ptr(r.row), nat.ptr(r.col), nat.ptr(r.kind), s)
        no = self.order + 1
        r.g = torch.empty((max(nref, 1), no), dtype=torch.float64, device=dev)
        r.f = torch.empty((max(nref, 1), 3, no), dtype=torch.float64, device=dev)
        nat.call("bem200_refine_integrals", nref, nat.ptr(r.row), nat.ptr(r.col), nat.ptr(r.kind),
                 nat.ptr(self.pos), nat.ptr(self.nvec), nat.ptr(self.tvec1), nat.ptr(self.tvec2),
                 nat.ptr(self.area), nat.ptr(self.nodes), nat.ptr(self.face_kind), nat.ptr(self.rules),
                 self.n28, self.n3, self.n4, self.order, nat.ptr(r.g), nat.ptr(r.f), s)
        self.corr = torch.zeros(n, dtype=torch.float64, device=dev)
        nat.call("bem200_closed_correction", n, self.npart, nat.ptr(self.pid), nat.ptr(self.closed_mask),
                 nat.ptr(self.pos), nat.ptr(self.nvec), nat.ptr(self.area), nref, nat.ptr(row_ptr), nat.ptr(r.row),
                 nat.ptr(r.col), nat.ptr(r.kind), self.order, nat.ptr(r.f), nat.ptr(self.corr), s)
        r.fn = torch.empty((max(nref, 1), no), dtype=torch.float64, device=dev)
        nat.call("bem200_refine_project", nref, nat.ptr(r.row), nat.ptr(self.nvec), self.order, nat.ptr(r.f),
                 nat.ptr(r.fn), s)
        self.refined = r

    # --------------------------------------------------------- evaluation
    def wavenumbers(self, enei):
        ks = []
        for m in self.p1.eps:
            k = complex(np.asarray(m(enei)[1]).ravel()[0])
            ks.append(k)
        return ks

    def _blk_mat(self, terms):
        """terms: 4 region pairs (or None) for slots (G1+, G1-, G2+, G2-)."""
        torch = _torch()
        npart = self.npart
        bm = np.zeros((npart, npart, 4), dtype=np.int32)
        for slot, rp in enumerate(terms):
            if rp is not None:
                bm[:, :, slot] = self.con[rp[0]][rp[1]]
        return torch.as_tensor(bm.reshape(-1), device=self.device)

    def assemble(self, enei, terms, dtype="c128", outputs=(True, True, True, True), out=None):
        """Run the fused assembly kernel; returns [G1, G2, H1, H2] (None where not requested)."""
        torch = _torch()
        ks = self.wavenumbers(enei)
        kmat = (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])
        tdt = torch.complex128 if dtype == "c128" else torch.complex64
        code = nat.C128 if dtype == "c128" else nat.C64
        n = self.n
        if out is None:
            out = [torch.empty((n, n), dtype=tdt, device=self.device) if want else None for want in outputs]
        blk = self._blk_mat(terms)
        r = self.refined
        nat.call("bem200_green_assemble", n, self.npart, nat.ptr(self.pid), nat.ptr(blk), len(ks),
                 ctypes.cast(kmat, ctypes.c_void_p), nat.ptr(self.pos), nat.ptr(self.nvec), nat.ptr(self.area),
                 r.nref, nat.ptr(r.row), nat.ptr(r.col), self.order, nat.ptr(r.g), nat.ptr(r.fn), code,
                 nat.ptr(out[0]), nat.ptr(out[1]), nat.ptr(out[2]), nat.ptr(out[3]), n, nat.stream_ptr())
        return out

    def bem_matrices(self, enei, dtype="c128", out=None):
        """G1 = G11 - G21, G2 = G22 - G12, H1 = H1_11 - H1_21, H2 = H2_22 - H2_12
        (reference mnpbem/bem/bem_ret.py:407-423) as device tensors."""
        return self.assemble(enei, [(0, 0), (1, 0), (1, 1), (0, 1)], dtype=dtype, out=out)

    def eval(self, i, j, key, enei, ind=None, as_tensor=False):
        """One region-pair matrix (reference CompGreenRet.eval, compgreen_ret.py:507).

        Keys G, F, H1, H2 give (n, n) matrices; Gp, H1p, H2p the Cartesian
        derivatives as (n, 3, n) arrays (reference layout).  Returns a host
        numpy array (or the device tensor when ``as_tensor``), or the int 0
        when region i of no particle connects to region j.
        """
        if ind is not None:
            raise NotImplementedError("CompGreenRet.eval: element selection (ind) is not supported")
        if key not in ("G", "F", "H1", "H2", "Gp", "H1p", "H2p"):
            raise ValueError("Unknown key: {}".format(key))
        if not np.any(self.con[i][j] > 0):
            return 0
        if key in ("Gp", "H1p", "H2p"):
            M = self.eval_cart(i, j, key, enei)
        elif key == "G":
            M = self.assemble(enei, [(i, j), None, None, None], outputs=(True, False, False, False))[0]
        elif key in ("H1", "F"):
            M = self.assemble(enei, [(i, j), None, None, None], outputs=(False, False, True, False))[2]
            if key == "F":
                self._sub_diag(M, (i, j), 2 * np.pi)
        else:
            M = self.assemble(enei, [None, None, (i, j), None], outputs=(False, False, False, True))[3]
        return M if as_tensor else M.cpu().numpy()

    def _kmat(self, enei):
        ks = self.wavenumbers(enei)
        return len(ks), (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])

    def _con_table(self, i, j):
        torch = _torch()
        return torch.as_tensor(np.ascontiguousarray(self.con[i][j], dtype=np.int32).reshape(-1), device=self.device)

    def eval_cart(self, i, j, key, enei):
        """Gp, H1p or H2p of region pair (i, j) as an (n, 3, n) complex128
        device tensor (reference greenret_refined.py:812-864, assembled per
        particle block as compgreen_ret.py:811-858 does)."""
        torch = _torch()
        n = self.n
        nmat, kmat = self._kmat(enei)
        out = torch.empty((n, 3, n), dtype=torch.complex128, device=self.device)
        r = self.refined
        blk = self._con_table(i, j)
        nat.call("bem200_green_assemble_cart", n, self.npart, nat.ptr(self.pid), nat.ptr(blk), nmat,
                 ctypes.cast(kmat, ctypes.c_void_p), nat.ptr(self.pos), nat.ptr(self.nvec), nat.ptr(self.area),
                 r.nref, nat.ptr(r.row), nat.ptr(r.col), self.order, nat.ptr(r.f),
                 {"Gp": 0, "H1p": 1, "H2p": 2}[key], nat.ptr(out), nat.stream_ptr())
        return out

    def _solution_device(self, sig):
        """sig1, sig2 (n, p) and h1, h2 (n, 3, p) of a solution as complex128
        device tensors, and p."""
        torch = _torch()
        n = self.n
        vals = [np.asarray(getattr(sig, k)) for k in ("sig1", "sig2", "h1", "h2")]
        npol = 1 if vals[0].ndim == 1 else vals[0].shape[1]
        out = []
        for k, v in enumerate(vals):
            shape = (n, npol) if k < 2 else (n, 3, npol)
            out.append(torch.as_tensor(np.ascontiguousarray(v.reshape(shape)), dtype=torch.complex128,
                                       device=self.device))
        return out, npol

    def _apply(self, sig, inout, field):
        torch = _torch()
        if inout not in (1, 2):
            raise ValueError("inout must be 1 (inside) or 2 (outside)")
        n = self.n
        r = self.refined
        reg = min(inout - 1, len(self.con) - 1)
        (s1, s2, h1, h2), npol = self._solution_device(sig)
        nmat, kmat = self._kmat(sig.enei)
        blk0, blk1 = self._con_table(reg, 0), self._con_table(reg, 1)
        cdt = dict(dtype=torch.complex128, device=self.device)
        common = [n, self.npart, nat.ptr(self.pid), nat.ptr(blk0), nat.ptr(blk1), nmat,
                  ctypes.cast(kmat, ctypes.c_void_p), nat.ptr(self.pos), nat.ptr(self.nvec), nat.ptr(self.area),
                  nat.ptr(r.row_ptr) if r.nref > 0 else None, nat.ptr(r.col), self.order, nat.ptr(r.g)]
        if field:
            e = torch.empty((n, 3, npol), **cdt)
            hh = torch.empty((n, 3, npol), **cdt)
            nat.call("bem200_green_field", *common, nat.ptr(r.f), inout, 2 * np.pi / sig.enei, npol, nat.ptr(s1),
                     nat.ptr(s2), nat.ptr(h1), nat.ptr(h2), nat.ptr(e), nat.ptr(hh), nat.stream_ptr())
            return [e, hh], npol
        phi = torch.empty((n, npol), **cdt)
        phip = torch.empty((n, npol), **cdt)
        a = torch.empty((n, 3, npol), **cdt)
        ap = torch.empty((n, 3, npol), **cdt)
        nat.call("bem200_green_potential", *common, nat.ptr(r.fn), inout, npol, nat.ptr(s1), nat.ptr(s2),
                 nat.ptr(h1), nat.ptr(h2), nat.ptr(phi), nat.ptr(phip), nat.ptr(a), nat.ptr(ap), nat.stream_ptr())
        return [phi, phip, a, ap], npol

    def potential(self, sig, inout=1):
        """Potentials and surface derivatives of solution ``sig`` inside
        (inout=1) or outside (inout=2) of the surface (reference
        CompGreenRet.potential, compgreen_ret.py:976-1038):
        phi = G sig1 + G sig2, phip = H sig1 + H sig2, a = G h1 + G h2,
        ap = H h1 + H h2 with the Green functions of region pairs
        (inout, 1) and (inout, 2) and H = H1 (inside) or H2 (outside).
        Returns a CompStruct with phi1, phi1p, a1, a1p (or phi2 ...)."""
        from .planewave import CompStruct
        (phi, phip, a, ap), npol = self._apply(sig, inout, field=False)
        phi, phip, a, ap = [t.cpu().numpy() for t in (phi, phip, a, ap)]
        if npol == 1:
            phi, phip, a, ap = phi[:, 0], phip[:, 0], a[:, :, 0], ap[:, :, 0]
        sfx = str(inout)
        return CompStruct(self.p1, sig.enei, **{"phi" + sfx: phi, "phi" + sfx + "p": phip, "a" + sfx: a,
                                               "a" + sfx + "p": ap})

    def field(self, sig, inout=1):
        """Electric and magnetic fields of solution ``sig`` at the faces, inside
        (inout=1) or outside (inout=2) (reference CompGreenRet.field,
        compgreen_ret.py:912-974): e = i k (G h1 + G h2) - Hp sig1 - Hp sig2,
        h = Hp x h1 + Hp x h2 with Hp = H1p (inside) or H2p (outside).
        Returns a CompStruct with e and h ((n, 3) or (n, 3, npol))."""
        from .planewave import CompStruct
        (e, h), npol = self._apply(sig, inout, field=True)
        e, h = e.cpu().numpy(), h.cpu().numpy()
        if npol == 1:
            e, h = e[:, :, 0], h[:, :, 0]
        return CompStruct(self.p1, sig.enei, e=e, h=h)

    def _sub_diag(self, M, rp, val):
        torch = _torch()
        con = self.con[rp[0]][rp[1]]
        off = self.p1.offsets
        for a in range(self.npart):
            if con[a, a] > 0:
                idx = torch.arange(int(off[a]), int(off[a + 1]), device=self.device)
                M[idx, idx] -= val
