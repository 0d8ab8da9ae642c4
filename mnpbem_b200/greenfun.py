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

        Returns a host numpy array (or the device tensor when ``as_tensor``),
        or the int 0 when region i of no particle connects to region j.
        """
        if ind is not None:
            raise NotImplementedError("CompGreenRet.eval: element selection (ind) is not supported")
        if key not in ("G", "F", "H1", "H2"):
            raise NotImplementedError("CompGreenRet.eval: key {!r} is not supported".format(key))
        if not np.any(self.con[i][j] > 0):
            return 0
        if key == "G":
            M = self.assemble(enei, [(i, j), None, None, None], outputs=(True, False, False, False))[0]
        elif key in ("H1", "F"):
            M = self.assemble(enei, [(i, j), None, None, None], outputs=(False, False, True, False))[2]
            if key == "F":
                self._sub_diag(M, (i, j), 2 * np.pi)
        else:
            M = self.assemble(enei, [None, None, (i, j), None], outputs=(False, False, False, True))[3]
        return M if as_tensor else M.cpu().numpy()

    def _sub_diag(self, M, rp, val):
        torch = _torch()
        con = self.con[rp[0]][rp[1]]
        off = self.p1.offsets
        for a in range(self.npart):
            if con[a, a] > 0:
                idx = torch.arange(int(off[a]), int(off[a + 1]), device=self.device)
                M[idx, idx] -= val
