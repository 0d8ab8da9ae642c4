"""Iterative retarded BEM solver on the GPU -- drop-in for the reference ``BEMRetIter``.

``BEMRetIter(p, **options).solve(exc)`` returns ``(sig, self)`` like
mnpbem/bem/bem_ret_iter.py:1636-1744: restarted GMRES on the 8 n p packed
system of Garcia de Abajo & Howie (phi, a, alpha, De) with

* the matrix-vector product ``A x`` = the full BEM operator applied in FP64
  (``bem200_bem_apply``: G1, G2, H1, H2 in complex128 -- reference
  ``_afun``, bem_ret_iter.py:1362-1501), or the H-matrix product when
  ``hmatrix=True`` (``mnpbem_b200.hmatrix``);
* the preconditioner ``M`` (``precond='hmat'``, the reference default) = one
  solve with the factored dense BEM (reference ``_mfun``, :1503-1634).  The
  factors are complex64 built on tcgen05 tensor cores
  (``precond_precision='mixed'``, default) or complex128 (``'fp64'``);
  ``precond=None`` runs unpreconditioned GMRES, with M = I pairing phi, a,
  De, alpha with sig1, h1, sig2, h2 as the reference's packed vectors do.

GMRES is right-preconditioned (A M u = b, x = M u), so ``tol`` bounds the true
relative residual ||b - A x|| / ||b||, the quantity the reference reports.
Orthogonalisation (CGS2), basis combinations and the operator run in
libbem200 kernels; only the (restart + 1) x restart Hessenberg least-squares
problem is solved on the host.
"""
import ctypes

import numpy as np

from . import _native as nat
from .bem import BEMRet, _ENGINES
from .planewave import CompStruct


def _torch():
    import torch
    return torch


class GMRESResult:
    """Outcome of one GMRES solve: flag (0 converged, 1 not), iter, relres."""

    def __init__(self, flag, iters, relres, history):
        self.flag = flag
        self.iter = iters
        self.relres = relres
        self.history = history


def gmres(apply_A, apply_M, b, tol=1e-4, maxit=200, restart=None):
    """Restarted, right-preconditioned GMRES on device vectors (complex128).

    apply_A(x, out) writes A x into ``out``; apply_M(v, out) writes M v (None:
    M = I).  b: device vector.  Returns (x, GMRESResult).  The iteration
    stops when ||b - A x|| <= tol ||b|| or after ``maxit`` matrix products
    (the reference's scipy ``gmres`` with ``restart`` defaulting to
    ``maxit``, mnpbem/bem/bem_iter.py:86-90).  Givens rotations use a real
    cosine: [c s; -conj(s) c] [a; b] = [r; 0].
    """
    torch = _torch()
    L = nat.lib()
    s = nat.stream_ptr()
    ln = b.numel()
    m = int(restart) if restart is not None else int(maxit)
    m = max(1, min(m, int(maxit), ln))
    dev = b.device
    V = torch.empty((m + 1, ln), dtype=torch.complex128, device=dev)
    z = torch.empty(ln, dtype=torch.complex128, device=dev) if apply_M is not None else None
    u = torch.empty(ln, dtype=torch.complex128, device=dev)
    r = torch.empty(ln, dtype=torch.complex128, device=dev)
    x = torch.zeros(ln, dtype=torch.complex128, device=dev)
    scr = torch.empty(int(L.bem200_gmres_orth_workspace_size(m)), dtype=torch.uint8, device=dev)
    ydev = torch.empty(16 * (m + 1), dtype=torch.uint8, device=dev)
    hbuf = (ctypes.c_double * (2 * (m + 1) + 1))()
    one = (ctypes.c_double * 2)(1.0, 0.0)
    mone = (ctypes.c_double * 2)(-1.0, 0.0)

    def orth(j):
        nat.call("bem200_gmres_orth", ln, j, nat.ptr(V), hbuf, nat.ptr(scr), s)
        h = np.frombuffer(hbuf, dtype=np.float64, count=2 * (j + 1) + 1)
        return h[0:2 * (j + 1):2] + 1j * h[1:2 * (j + 1):2], float(h[2 * (j + 1)])

    r.copy_(b)
    V[0].copy_(r)
    _, bnorm = orth(-1)
    history = []
    if not (bnorm > 0):
        return x, GMRESResult(0, 0, 0.0, [0.0])
    rnorm = bnorm
    total = 0
    flag = 1
    while True:
        history.append(rnorm / bnorm)
        if rnorm <= tol * bnorm:
            flag = 0
            break
        if total >= maxit:
            break
        H = np.zeros((m + 1, m), dtype=complex)
        cs = np.zeros(m)
        sn = np.zeros(m, dtype=complex)
        g = np.zeros(m + 1, dtype=complex)
        g[0] = rnorm
        k = 0
        for j in range(m):
            if apply_M is not None:
                apply_M(V[j], z)
                apply_A(z, V[j + 1])
            else:
                apply_A(V[j], V[j + 1])
            hcol, hn = orth(j)
            total += 1
            col = np.concatenate([hcol, [hn]]).astype(complex)
            for i in range(j):
                t = cs[i] * col[i] + sn[i] * col[i + 1]
                col[i + 1] = -np.conj(sn[i]) * col[i] + cs[i] * col[i + 1]
                col[i] = t
            a_, b_ = col[j], col[j + 1]
            den = np.hypot(abs(a_), abs(b_))
            if den == 0:
                cs[j], sn[j] = 1.0, 0.0
            elif abs(a_) == 0:
                cs[j], sn[j] = 0.0, 1.0
            else:
                cs[j] = abs(a_) / den
                sn[j] = (a_ / abs(a_)) * np.conj(b_) / den
            col[j] = cs[j] * a_ + sn[j] * b_
            col[j + 1] = 0.0
            H[:j + 2, j] = col[:j + 2]
            g[j + 1] = -np.conj(sn[j]) * g[j]
            g[j] = cs[j] * g[j]
            k = j + 1
            if abs(g[j + 1]) <= tol * bnorm or total >= maxit or hn == 0:
                break
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        ybuf = np.ascontiguousarray(np.stack([y.real, y.imag], axis=1).ravel())
        nat.call("bem200_gmres_combine", ln, k, nat.ptr(V), ybuf.ctypes.data_as(ctypes.c_void_p), nat.ptr(u),
                 nat.ptr(ydev), s)
        if apply_M is not None:
            apply_M(u, z)
            nat.call("bem200_zaxpy", ln, one, nat.ptr(z), nat.ptr(x), s)
        else:
            nat.call("bem200_zaxpy", ln, one, nat.ptr(u), nat.ptr(x), s)
        # true residual r = b - A x
        apply_A(x, u)
        r.copy_(b)
        nat.call("bem200_zaxpy", ln, mone, nat.ptr(u), nat.ptr(r), s)
        V[0].copy_(r)
        _, rnorm = orth(-1)
    return x, GMRESResult(flag, total, rnorm / bnorm, history)


class BEMRetIter:
    """Iterative retarded BEM solver (reference class mnpbem/bem/bem_ret_iter.py:455).

    Options (reference defaults): solver='gmres', tol=1e-4, maxit=200,
    restart=None (= maxit), precond='hmat' (dense BEM factors as M) or None,
    output=0; hmatrix=False (True: H-matrix operator, htol=1e-6,
    kmax=[4, 100], cleaf=200, eta=2.5); B200 options: precond_precision
    ('mixed' | 'fp64'), engine ('bf16x3' | 'simt'), hmat_fill ('auto':
    compress the dense matrices the mixed preconditioner keeps, otherwise
    compute every stored H-matrix entry on demand from the Green function;
    'green' | 'dense' force one way).
    """

    name = "bemsolver"
    needs = {"sim": "ret"}

    def __init__(self, p, enei=None, solver="gmres", tol=1e-4, maxit=200, restart=None, precond="hmat", output=0,
                 hmatrix=False, htol=1e-6, kmax=(4, 100), cleaf=200, eta=2.5, precond_precision="mixed",
                 engine="bf16x3", hmat_fill="auto", **options):
        torch = _torch()
        if p is None:
            raise ValueError("BEMRetIter: 'p' must be a ComParticle (or compatible particle object), got None.")
        if not (hasattr(p, "pos") and hasattr(p, "nvec") and hasattr(p, "eps")):
            raise TypeError("BEMRetIter: 'p' must expose ComParticle-like attributes (pos, nvec, eps); got {!r}."
                            .format(type(p).__name__))
        if solver in ("cgs", "bicgstab"):
            raise NotImplementedError("BEMRetIter: only solver='gmres' runs on the GPU")
        if solver != "gmres":
            raise ValueError("[error] iterative solver not known: <{}>".format(solver))
        if precond not in ("hmat", None):
            raise ValueError("BEMRetIter: precond must be 'hmat' or None")
        if hmat_fill not in ("auto", "green", "dense"):
            raise ValueError("BEMRetIter: hmat_fill must be 'auto', 'green' or 'dense'")
        if not torch.cuda.is_available():
            raise RuntimeError("BEMRetIter: a CUDA device is required (no CPU fallback)")
        self.p = p
        self.hmat_fill = hmat_fill
        self.solver = solver
        self.tol = float(tol)
        self.maxit = int(maxit)
        self.restart = restart
        self.precond = precond
        self.output = output
        self.hmatrix = bool(hmatrix)
        self.htol = float(htol)
        self.kmax = kmax
        self.cleaf = int(cleaf)
        self.eta = float(eta)
        self.options = dict(options)
        self.enei = None
        self.dev = torch.device("cuda")
        self.n = p.n
        # the dense BEM solver supplies the Green assembly, the eps handling
        # and (when preconditioning) the factors
        self._bem = BEMRet(p, precision=precond_precision, engine=engine, **options)
        self.g = self._bem.g
        self._G = None       # complex128 G1, G2, H1, H2 for the operator
        self._hmat = None    # H-matrix operator (hmatrix=True)
        self._flag, self._relres, self._iter = [], [], []
        if enei is not None:
            self.init(enei)

    # ----------------------------------------------------------------- init
    def init(self, enei):
        """Operator (and preconditioner factors) at wavelength ``enei`` (nm)."""
        if self.enei is not None and np.isclose(self.enei, enei):
            return self
        torch = _torch()
        bem = self._bem
        n = self.n
        if self.precond is not None:
            bem.clear()
            bem.init(enei)
            self._eps_args = (bem._eps_mode, bem._e1p, bem._e2p)
        else:
            bem.k = 2 * np.pi / enei
            bem._eps(enei)
            self._eps_args = (bem._eps_mode, bem._e1p, bem._e2p)
        self.k = 2 * np.pi / enei
        if self.hmatrix:
            from .hmatrix import BEMHMatrices
            if self._hmat is None:
                self._hmat = BEMHMatrices(self.p, self.g, htol=self.htol, kmax=self.kmax, cleaf=self.cleaf,
                                          eta=self.eta)
            # 'auto': reuse the dense matrices the mixed preconditioner keeps, else
            # compute the stored entries on demand; 'green' / 'dense' force one way
            have = self.precond is not None and bem._prec == 1
            shared = bem._G128 if (have and self.hmat_fill != "green") else None
            self._hmat.build(enei, mats=shared, fill="dense" if self.hmat_fill == "dense" else "green")
        else:
            if bem._prec == 1 and self.precond is not None:
                self._G = bem._G128  # assembled by the mixed init
            else:
                if self._G is None:
                    self._G = [torch.empty((n, n), dtype=torch.complex128, device=self.dev) for _ in range(4)]
                self.g.bem_matrices(enei, dtype="c128", out=self._G)
        self.enei = enei
        return self

    __call__ = init

    def clear(self):
        self.enei = None
        return self

    # ------------------------------------------------------------- operators
    def _apply_A(self, npol):
        torch = _torch()
        n = self.n
        L = nat.lib()
        scr = torch.empty(int(L.bem200_bem_apply_workspace_size(n, npol)), dtype=torch.uint8, device=self.dev)
        em, e1, e2 = self._eps_args
        nv = self._bem._nvec
        k = self.k
        np_ = n * npol

        if self.hmatrix:
            hm = self._hmat

            def apply(x, out):
                hm.apply(npol, em, e1, e2, nv, k, x, out)
            return apply
        G = self._G

        def apply(x, out):
            base = x.data_ptr()
            nat.call("bem200_bem_apply", n, npol, nat.ptr(G[0]), nat.ptr(G[1]), nat.ptr(G[2]), nat.ptr(G[3]), em,
                     e1, e2, nat.ptr(nv), k, ctypes.c_void_p(base), ctypes.c_void_p(base + 16 * 4 * np_), None,
                     nat.ptr(out), nat.ptr(scr), nat.stream_ptr())
        return apply

    def _apply_M(self, npol):
        if self.precond is None:
            n = self.n

            def relabel(v, out):  # M = I with the reference's pairing of the two spaces
                nat.call("bem200_bem_relabel", n, npol, nat.ptr(v), nat.ptr(out), nat.stream_ptr())
            return relabel
        torch = _torch()
        bem = self._bem
        L = nat.lib()
        scr = torch.empty(int(L.bem200_bem_solve_workspace_size(bem._prec, self.n, npol)), dtype=torch.uint8,
                          device=self.dev)
        em, e1, e2 = self._eps_args

        def apply(v, out):
            nat.call("bem200_bem_precond", bem._cprec, _ENGINES[bem.engine], self.n, npol, nat.ptr(bem._ws),
                     nat.ptr(v), em, e1, e2, nat.ptr(bem._nvec), self.k, nat.ptr(out), nat.ptr(scr),
                     nat.ptr(bem._gws), bem._gws_bytes, nat.stream_ptr())
        return apply

    # ----------------------------------------------------------------- solve
    def solve_device(self, bt, npol):
        """GMRES for a device right-hand side (8 n npol complex128, layout of
        ``BEMRet.rhs``); returns (W1, W2) device tensors like BEMRet.solve_device."""
        n = self.n
        x, res = gmres(self._apply_A(npol), self._apply_M(npol), bt, tol=self.tol, maxit=self.maxit,
                       restart=self.restart)
        self._flag.append(res.flag)
        self._relres.append(res.relres)
        self._iter.append(res.iter)
        self.last = res
        if self.output:
            print("gmres({}): iter {}, relres {:.3e}, flag {}".format(self.restart or self.maxit, res.iter,
                                                                     res.relres, res.flag))
        W = x.view(2, n, 4 * npol)
        return W[0], W[1]

    def solve(self, exc):
        """Surface charges and currents for excitation ``exc``; returns (sig, self)."""
        torch = _torch()
        enei = exc["enei"] if not hasattr(exc, "enei") else exc.enei
        self.init(enei)
        b, npol = self._bem.rhs(exc)
        n = self.n
        bt = torch.as_tensor(b, dtype=torch.complex128).to(self.dev)
        W1, W2 = self.solve_device(bt, npol)
        w1 = W1.cpu().numpy()
        w2 = W2.cpu().numpy()
        sig1, h1 = w1[:, :npol], w1[:, npol:].reshape(n, 3, npol)
        sig2, h2 = w2[:, :npol], w2[:, npol:].reshape(n, 3, npol)
        if npol == 1:
            sig1, sig2, h1, h2 = sig1[:, 0], sig2[:, 0], h1[:, :, 0], h2[:, :, 0]
        sig = CompStruct(self.p, enei, sig1=sig1, sig2=sig2, h1=h1, h2=h2)
        return sig, self

    def __truediv__(self, exc):
        return self.solve(exc)[0]

    def info(self):
        """(iterations, relative residuals, flags) of the solves so far
        (reference BEMIter.info, mnpbem/bem/bem_iter.py:191)."""
        return list(self._iter), list(self._relres), list(self._flag)
