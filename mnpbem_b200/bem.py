"""Dense retarded BEM solver on the GPU -- drop-in for the reference ``BEMRet``.

``BEMRet(p).solve(exc)`` returns ``(sig, self)`` with ``sig.sig1, sig2, h1,
h2`` as host numpy arrays, exactly like mnpbem/bem/bem_ret.py:1569-1831.
Everything per wavelength runs in libbem200 on the GPU:

* ``precision='fp64'`` (default): complex128 assembly, LU factors, Sigma /
  Delta build and the Eq. (19, 20) solve -- the drop-in path;
* ``precision='mixed'``: complex64 factors built with tcgen05 tensor-core
  GEMMs (``engine='bf16x3'``; ``'simt'`` uses CUDA cores),
  then iterative refinement against the complex128 BEM operator until the
  max-norm residual drops below ``ir_tol`` times the right-hand side.
  Refinement whose sweeps stop contracting (the contraction rate of
  refinement is about cond(A) times the complex64 rounding error, so a slow
  or diverging sweep is the condition estimate that the factors are not good
  enough) continues as GMRES-IR: restarted GMRES on the FP64 operator,
  right-preconditioned by the same complex64 factors (``gmres_ir=True``).
  A solve that still misses ``ir_tol`` raises ``RuntimeError``.

There is no CPU fallback: without a GPU or the library, construction raises.
"""
import ctypes

import numpy as np

from . import _native as nat
from .greenfun import CompGreenRet
from .planewave import CompStruct

_ENGINES = {"simt": 0, "bf16x3": 1}


def _torch():
    import torch
    return torch


def _excitation_rhs(p, exc, enei):
    """phi, a, alpha, De (Eqs. 10, 11, 15, 18) with a trailing polarisation axis.

    Reference: mnpbem/bem/bem_ret.py:1360-1429 (MATLAB excitation.m:21-29).
    """
    n = p.n

    def field(name):
        v = exc.get(name, 0) if hasattr(exc, "get") else exc[name]
        return None if (v is None or (np.isscalar(v) and v == 0)) else np.asarray(v, dtype=complex)

    f = {k: field(k) for k in ("phi1", "phi1p", "phi2", "phi2p", "a1", "a1p", "a2", "a2p")}
    npol = 1
    for k in ("a1", "a2", "a1p", "a2p"):
        if f[k] is not None and f[k].ndim == 3:
            npol = f[k].shape[2]
    for k in ("phi1", "phi2", "phi1p", "phi2p"):
        if f[k] is not None and f[k].ndim == 2:
            npol = max(npol, f[k].shape[1])

    def s(v):  # scalar-like field -> (n, p)
        return np.zeros((n, npol), complex) if v is None else np.broadcast_to(v.reshape(n, -1), (n, npol))

    def vec(v):  # vector field -> (n, 3, p)
        return np.zeros((n, 3, npol), complex) if v is None else np.broadcast_to(v.reshape(n, 3, -1), (n, 3, npol))

    k = 2 * np.pi / enei
    e1 = p.eps1(enei)[:, None]
    e2 = p.eps2(enei)[:, None]
    nv = p.nvec
    phi1, phi2, phi1p, phi2p = s(f["phi1"]), s(f["phi2"]), s(f["phi1p"]), s(f["phi2p"])
    a1, a2, a1p, a2p = vec(f["a1"]), vec(f["a2"]), vec(f["a1p"]), vec(f["a2p"])
    phi = phi2 - phi1
    a = a2 - a1
    alpha = (a2p - a1p) - 1j * k * (nv[:, :, None] * (phi2 * e2)[:, None, :] - nv[:, :, None] * (phi1 * e1)[:, None, :])
    De = (e2 * phi2p - e1 * phi1p) - 1j * k * (np.einsum("ij,ijk->ik", nv, a2) * e2
                                                - np.einsum("ij,ijk->ik", nv, a1) * e1)
    return npol, phi, a, alpha, De


_DIAGONAL_PIVOTS = 4  # BEM200_GETRF_DIAGONAL_PIVOTS


class BEMRet:
    """Retarded BEM solver (reference class mnpbem/bem/bem_ret.py:138)."""

    name = "bemsolver"
    needs = {"sim": "ret"}

    def __init__(self, p, enei=None, precision="fp64", engine="bf16x3", ir_tol=1e-12, ir_maxit=30, gmres_ir=True,
                 gmres_maxit=200, lu_tiles=None, pivoting="auto", explicit_inverses=True, **options):
        torch = _torch()
        if p is None:
            raise ValueError("BEMRet: 'p' must be a ComParticle (or compatible particle object), got None.")
        if not (hasattr(p, "pos") and hasattr(p, "nvec") and hasattr(p, "eps")):
            raise TypeError("BEMRet: 'p' must expose ComParticle-like attributes (pos, nvec, eps); got {!r}."
                            .format(type(p).__name__))
        if precision not in ("fp64", "mixed"):
            raise ValueError("BEMRet: precision must be 'fp64' or 'mixed'")
        if engine not in _ENGINES:
            raise ValueError("BEMRet: engine must be one of {}".format(sorted(_ENGINES)))
        if not torch.cuda.is_available():
            raise RuntimeError("BEMRet: a CUDA device is required (no CPU fallback)")
        self.p = p
        self.precision = precision
        self.engine = engine if precision == "mixed" else "simt"
        self.ir_tol = float(ir_tol)
        self.ir_maxit = int(ir_maxit)
        self.gmres_ir = bool(gmres_ir)
        self.gmres_maxit = int(gmres_maxit)
        if not (lu_tiles is None or lu_tiles == "auto" or (isinstance(lu_tiles, int) and lu_tiles % 32 == 0
                                                           and 64 <= lu_tiles <= 1024)):
            raise ValueError("BEMRet: lu_tiles must be None, 'auto' or a look-ahead width (multiple of 32, 64-1024)")
        self.lu_tiles = lu_tiles
        # "auto": LUs without the pivot search, checked against partial
        # pivoting's choice, repeated with partial pivoting when a factor
        # matrix needs row exchanges; "partial": always partial pivoting
        if pivoting not in ("auto", "partial"):
            raise ValueError("BEMRet: pivoting must be 'auto' or 'partial'")
        self.pivoting = pivoting
        # mixed precision with pivoting='auto': the complex64 factors are first
        # built as explicit inverses (G1^-1, G2^-1, Delta^-1, Sigma^-1 without
        # pivoting, probe-checked), so that every refinement sweep is a few
        # matrix products; if a check fails, LU factors as above
        self.explicit_inverses = bool(explicit_inverses)
        self.last_pivoting = None
        # stage timer of init (profiling): set to (ctypes.c_float * 4)() to record the phases
        self._phase_buf = None
        self.last_init_phases_ms = None
        self.options = dict(options)
        self.enei = None
        self.dev = torch.device("cuda")
        self.g = CompGreenRet(p, p, **self.options)
        n = self.n = p.n
        prec = 0 if precision == "fp64" else 1
        self._prec = prec
        # precision code of the factors in the workspace for the library
        # calls: 0 fp64, 1 mixed with LU factors, 2 mixed with explicit inverses
        self._cprec = prec
        self._ws = None      # factor workspaces, allocated by the first init()
        self._nvec = torch.as_tensor(np.ascontiguousarray(p.nvec), dtype=torch.float64, device=self.dev)
        self.last_ir = None
        if enei is not None:
            self.init(enei)

    def _alloc(self):
        """Workspaces of the factors: 7 n x n slots, the GEMM operand space and,
        for the mixed path, the complex128 matrices of the FP64 operator.  Users
        that never factor (the unpreconditioned iterative solver) never pay for
        them."""
        if self._ws is not None:
            return
        torch = _torch()
        n, prec = self.n, self._prec
        L = nat.lib()
        self._ws = torch.empty(int(L.bem200_bem_workspace_size(prec, n)), dtype=torch.uint8, device=self.dev)
        slots = [ctypes.c_void_p() for _ in range(4)]
        nat.call("bem200_bem_slots", prec, n, nat.ptr(self._ws), *[ctypes.byref(s) for s in slots])
        self._slots = [s.value for s in slots]
        # operand space of the largest GEMM plus headroom for the concurrent
        # halves of the factor chains (each needs about a quarter of it)
        gbytes = int(L.bem200_gemm_workspace_size(_ENGINES[self.engine], n, n, n) * 5 // 4)
        self._gws = torch.empty(max(gbytes, 1), dtype=torch.uint8, device=self.dev)
        self._gws_bytes = gbytes
        if prec == 1:
            self._G128 = [torch.empty((n, n), dtype=torch.complex128, device=self.dev) for _ in range(4)]

    # ----------------------------------------------------------------- eps
    def _eps(self, enei):
        e1 = self.p.eps1(enei)
        e2 = self.p.eps2(enei)
        if np.allclose(e1, e1[0]) and np.allclose(e2, e2[0]):
            self._eps_mode = 0
            self._e1 = (ctypes.c_double * 2)(e1[0].real, e1[0].imag)
            self._e2 = (ctypes.c_double * 2)(e2[0].real, e2[0].imag)
            self._e1p, self._e2p = ctypes.cast(self._e1, ctypes.c_void_p), ctypes.cast(self._e2, ctypes.c_void_p)
        else:
            torch = _torch()
            if np.any(self.g.con[0][1] != 0):
                raise NotImplementedError("BEMRet: non-uniform eps with cross-connected regions (L = G eps G^-1)")
            self._eps_mode = 1
            self._d1 = torch.as_tensor(e1, dtype=torch.complex128, device=self.dev)
            self._d2 = torch.as_tensor(e2, dtype=torch.complex128, device=self.dev)
            self._e1p, self._e2p = nat.ptr(self._d1), nat.ptr(self._d2)

    # ---------------------------------------------------------------- init
    def init(self, enei):
        """Assemble G1, G2, H1, H2 and build the factors at wavelength ``enei`` (nm)
        (reference bem_ret.py:293-525).  Skipped if already initialised there."""
        if self.enei is not None and np.isclose(self.enei, enei):
            return self
        self._alloc()
        n = self.n
        self.k = 2 * np.pi / enei
        self._eps(enei)
        s = nat.stream_ptr()
        if self._prec == 1:
            self.g.bem_matrices(enei, dtype="c128", out=self._G128)
        if self.pivoting == "partial":
            modes = ["partial"]
        elif self._prec == 1 and self.explicit_inverses:
            modes = ["inverse", "diagonal", "partial"]
        else:
            modes = ["diagonal", "partial"]
        for mode in modes:
            cprec = 2 if mode == "inverse" else self._prec
            if self._prec == 0:
                self._assemble_into_slots(enei, "c128")
            else:
                for src, dst in zip(self._G128, self._slots):
                    nat.call("bem200_convert_c128_c64", n * n, nat.ptr(src), ctypes.c_void_p(dst), s)
            info = ctypes.c_int32(0)
            st = nat.lib().bem200_bem_init_ex(
                cprec, _ENGINES[self.engine], n, nat.ptr(self._ws), self._eps_mode, self._e1p, self._e2p,
                nat.ptr(self._nvec), self.k, nat.ptr(self._gws), self._gws_bytes,
                0 if mode == "partial" else _DIAGONAL_PIVOTS, self._lookahead(), self._phase_buf,
                ctypes.byref(info), s)
            if st == nat.ERR_PIVOTING and mode != "partial":
                continue  # a factor matrix needs row exchanges: the next, more general factorisation
            nat.check(st, "bem200_bem_init_ex")
            self.last_pivoting = mode
            self._cprec = cprec
            break
        if self._phase_buf is not None:
            self.last_init_phases_ms = list(self._phase_buf)
        self.enei = enei
        return self

    def _lookahead(self):
        """Look-ahead block width of the LU factorisations (0: the library's
        default); 'auto' measures it once per size on this GPU
        (mnpbem_b200.tuning, cached)."""
        if self.lu_tiles is None:
            return 0
        if self.lu_tiles == "auto":
            if getattr(self, "_la_tuned", None) is None:
                from .tuning import tune_lookahead
                self._la_tuned, _ = tune_lookahead(self.n, "c128" if self._prec == 0 else "c64",
                                                   _ENGINES[self.engine])
            return self._la_tuned
        return int(self.lu_tiles)

    def _assemble_into_slots(self, enei, dtype):
        g = self.g
        ks = g.wavenumbers(enei)
        kmat = (ctypes.c_double * (2 * len(ks)))(*[v for k in ks for v in (k.real, k.imag)])
        blk = g._blk_mat([(0, 0), (1, 0), (1, 1), (0, 1)])
        r = g.refined
        nat.call("bem200_green_assemble", self.n, g.npart, nat.ptr(g.pid), nat.ptr(blk), len(ks),
                 ctypes.cast(kmat, ctypes.c_void_p), nat.ptr(g.pos), nat.ptr(g.nvec), nat.ptr(g.area), r.nref,
                 nat.ptr(r.row), nat.ptr(r.col), g.order, nat.ptr(r.g), nat.ptr(r.fn),
                 nat.C128 if dtype == "c128" else nat.C64, *[ctypes.c_void_p(v) for v in self._slots], self.n,
                 nat.stream_ptr())

    __call__ = init

    # --------------------------------------------------------------- solve
    def rhs(self, exc):
        """Right-hand side b = [phi | a | alpha | De] (complex128, host) and npol."""
        enei = exc["enei"] if not hasattr(exc, "enei") else exc.enei
        npol, phi, a, alpha, De = _excitation_rhs(self.p, exc, enei)
        b = np.concatenate([phi.reshape(-1), a.reshape(-1), alpha.reshape(-1), De.reshape(-1)])
        return b, npol

    def solve_device(self, bt, npol):
        """Solve for a device right-hand side ``bt`` (8 n npol complex128); returns
        device tensors W1 = [sig1 | h1], W2 = [sig2 | h2] (n x 4 npol).  The
        factors of the current wavelength must be built (``init``)."""
        torch = _torch()
        n = self.n
        W1 = torch.empty((n, 4 * npol), dtype=torch.complex128, device=self.dev)
        W2 = torch.empty_like(W1)
        L = nat.lib()
        s = nat.stream_ptr()
        key = (npol,)
        if getattr(self, "_scratch_key", None) != key:
            self._scratch = torch.empty(int(L.bem200_bem_solve_workspace_size(self._prec, n, npol)),
                                        dtype=torch.uint8, device=self.dev)
            self._scratch_key = key
        scratch = self._scratch
        np_ = n * npol
        if self._prec == 0:
            base = bt.data_ptr()
            nat.call("bem200_bem_solve", 0, 0, n, npol, nat.ptr(self._ws), nat.ptr(bt),
                     ctypes.c_void_p(base + 16 * np_), ctypes.c_void_p(base + 16 * 4 * np_),
                     ctypes.c_void_p(base + 16 * 7 * np_), self._eps_mode, self._e1p, self._e2p,
                     nat.ptr(self._nvec), self.k, nat.ptr(W1), nat.ptr(W2), nat.ptr(scratch), nat.ptr(self._gws),
                     self._gws_bytes, s)
        else:
            it = ctypes.c_int32(0)
            rr = ctypes.c_double(0)
            G = self._G128
            st = L.bem200_bem_solve_ir_ex(self._cprec, _ENGINES[self.engine], n, npol, nat.ptr(self._ws),
                                          nat.ptr(G[0]), nat.ptr(G[1]), nat.ptr(G[2]), nat.ptr(G[3]), nat.ptr(bt),
                                          self._eps_mode, self._e1p, self._e2p, nat.ptr(self._nvec), self.k,
                                          self.ir_tol, self.ir_maxit, nat.ptr(W1), nat.ptr(W2), nat.ptr(scratch),
                                          nat.ptr(self._gws), self._gws_bytes, ctypes.byref(it), ctypes.byref(rr), s)
            self.last_ir = (int(it.value), float(rr.value), "ir")
            if st == nat.ERR_NOCONV and self.gmres_ir:
                W1, W2 = self._gmres_refine(bt, npol, W1, W2, int(it.value))
            else:
                nat.check(st, "bem200_bem_solve_ir")
        return W1, W2

    def _gmres_refine(self, bt, npol, W1, W2, sweeps):
        """GMRES-IR: continue a refinement that stopped contracting.  Solves
        A d = b - A x0 by restarted GMRES on the FP64 operator, right
        preconditioned by one solve with the complex64 factors, and returns
        x0 + d.  The tolerance is ``ir_tol`` on the 2-norm residual relative to
        ||b||; a miss raises RuntimeError."""
        torch = _torch()
        from .bem_iter import gmres
        n = self.n
        np_ = n * npol
        L = nat.lib()
        s = nat.stream_ptr()
        G = self._G128
        x0 = torch.cat([W1.reshape(-1), W2.reshape(-1)])
        ascr = torch.empty(int(L.bem200_bem_apply_workspace_size(n, npol)), dtype=torch.uint8, device=self.dev)
        pscr = torch.empty(int(L.bem200_bem_solve_workspace_size(1, n, npol)), dtype=torch.uint8, device=self.dev)

        def apply_A(v, out, b=None):
            nat.call("bem200_bem_apply", n, npol, nat.ptr(G[0]), nat.ptr(G[1]), nat.ptr(G[2]), nat.ptr(G[3]),
                     self._eps_mode, self._e1p, self._e2p, nat.ptr(self._nvec), self.k, nat.ptr(v),
                     ctypes.c_void_p(v.data_ptr() + 16 * 4 * np_), nat.ptr(b), nat.ptr(out), nat.ptr(ascr), s)

        def apply_M(v, out):
            nat.call("bem200_bem_precond", self._cprec, _ENGINES[self.engine], n, npol, nat.ptr(self._ws), nat.ptr(v),
                     self._eps_mode, self._e1p, self._e2p, nat.ptr(self._nvec), self.k, nat.ptr(out),
                     nat.ptr(pscr), nat.ptr(self._gws), self._gws_bytes, s)

        r0 = torch.empty_like(bt)
        apply_A(x0, r0, b=bt)
        bn = float(torch.linalg.vector_norm(bt))
        rn = float(torch.linalg.vector_norm(r0))
        if rn > self.ir_tol * bn:
            d, res = gmres(apply_A, apply_M, r0, tol=self.ir_tol * bn / rn, maxit=self.gmres_maxit,
                           restart=min(self.gmres_maxit, 50))
            x0 += d
            apply_A(x0, r0, b=bt)
            rn = float(torch.linalg.vector_norm(r0))
            self.last_ir = (sweeps, rn / bn, "gmres-ir", res.iter)
        else:
            self.last_ir = (sweeps, rn / bn, "gmres-ir", 0)
        if not (rn <= self.ir_tol * bn):
            raise RuntimeError("BEMRet: mixed-precision solve did not converge: {} refinement sweeps, then GMRES-IR "
                               "left the residual at {:.3e} of the right-hand side (ir_tol {:.1e})"
                               .format(sweeps, rn / bn, self.ir_tol))
        return x0[:4 * np_].view(n, 4 * npol), x0[4 * np_:].view(n, 4 * npol)

    def check_status(self):
        """Raise if a factor met a zero pivot or a bounded device wait gave up."""
        status = ctypes.c_int32(0)
        nat.call("bem200_bem_status", self._cprec, self.n, nat.ptr(self._ws), ctypes.byref(status),
                 nat.stream_ptr())
        if status.value != 0:
            raise RuntimeError("BEMRet: device status {} (3 = zero pivot in a factor, 5 = a bounded device wait "
                               "gave up)".format(status.value))

    def solve(self, exc):
        """Surface charges and currents for excitation ``exc``; returns (sig, self)
        (reference mnpbem/bem/bem_ret.py:1569-1831)."""
        torch = _torch()
        enei = exc["enei"] if not hasattr(exc, "enei") else exc.enei
        self.init(enei)
        b, npol = self.rhs(exc)
        n = self.n
        bt = torch.as_tensor(b, dtype=torch.complex128).to(self.dev, non_blocking=False)
        W1, W2 = self.solve_device(bt, npol)
        if self._prec == 0:
            self.check_status()
        w1 = W1.cpu().numpy()
        w2 = W2.cpu().numpy()
        sig1, h1 = w1[:, :npol], w1[:, npol:].reshape(n, 3, npol)
        sig2, h2 = w2[:, :npol], w2[:, npol:].reshape(n, 3, npol)
        if npol == 1:
            sig1, sig2, h1, h2 = sig1[:, 0], sig2[:, 0], h1[:, :, 0], h2[:, :, 0]
        sig = CompStruct(self.p, enei, sig1=sig1, sig2=sig2, h1=h1, h2=h2)
        return sig, self

    def cross_sections(self, exc, enei):
        """Extinction and scattering of a plane wave at ``enei`` with every
        per-wavelength step on the GPU: the right-hand side, the solve and the
        far fields; only the cross sections come back.  Returns dict ext, sca
        ((npol,) arrays)."""
        self.init(enei)
        bt, npol = exc.rhs_device(self.p, enei, self._eps_mode, self._e1p, self._e2p, device=self.dev)
        W1, W2 = self.solve_device(bt, npol)
        if self._prec == 0:
            self.check_status()
        ext, sca, _ = exc.cross_sections_device(self.p, enei, W1, W2)
        return {"ext": ext, "sca": sca}

    def __truediv__(self, exc):
        """``bem / exc`` -> sig (MATLAB ``bem \\ exc``)."""
        return self.solve(exc)[0]

    def clear(self):
        self.enei = None
        return self

    def potential(self, sig, inout=2):
        """Potentials and surface derivatives of a solution inside (inout=1) or
        outside (inout=2, default) of the particle surface (reference
        bem_ret.py:1833-1859, delegating to CompGreenRet.potential): phi, phip,
        a, ap computed on the GPU without storing the Green matrices (so no
        factorisation at sig.enei is needed)."""
        return self.g.potential(sig, inout)

    def field(self, sig, inout=2):
        """Electric and magnetic fields of a solution inside (inout=1) or
        outside (inout=2, default) of the particle surface (reference
        bem_ret.py:1861-1895, delegating to CompGreenRet.field with the
        Cartesian-derivative Green functions H1p / H2p), computed on the GPU
        without storing the Green matrices."""
        return self.g.field(sig, inout)
