"""GPU iterative solver (BEMRetIter: restarted GMRES on the 8 n packed BEM
system) against the CPU oracle's direct complex128 solve and its operator."""
import numpy as np
import pytest

from meshes import dimer, rel, sphere
from oracle import bem as obem
from oracle.pipeline import OracleBEM

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _iter(cp, enei, **kw):
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.bem_iter import BEMRetIter
    bem = BEMRetIter(cp, **kw)
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(cp, enei))
    return bem, sig, exc.extinction(sig), exc.scattering(sig)[0]


@pytest.mark.parametrize("mk,enei", [(sphere, 600.0), (dimer, 620.0)], ids=["sphere284", "dimer568"])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_preconditioned_gmres_matches_direct(cuda, mk, enei, prec):
    """precond='hmat': the dense factors precondition GMRES; a few iterations
    reach tol and the solution matches the direct FP64 solve."""
    cp = mk()
    bem, sig, ext, sca = _iter(cp, enei, tol=1e-11, precond_precision=prec)
    ref = OracleBEM(cp).solve(enei, POL, DIR)
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-11 and it[-1] <= 8, bem.info()
    assert abs(ext - ref["ext"][0]) / abs(ref["ext"][0]) < 1e-9
    assert abs(sca - ref["sca"][0]) / abs(ref["sca"][0]) < 1e-9
    assert rel(sig.sig2, ref["sig2"][:, 0]) < 1e-8
    assert rel(sig.h1, ref["h1"][:, :, 0]) < 1e-8


def test_unpreconditioned_gmres_default_tol(cuda):
    """precond=None at the reference defaults (tol 1e-4): the same Krylov
    iteration as the reference's scipy GMRES (oracle restatement with the
    reference's packing), so the iteration count, the true residual (oracle
    FP64 operator on the host) and the extinction agree with it."""
    from oracle import farfield as off
    cp = sphere()
    enei = 600.0
    bem, sig, ext, sca = _iter(cp, enei, precond=None, tol=1e-4, maxit=300)
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-4
    ob = OracleBEM(cp)
    G1, G2, H1, H2 = ob.matrices(enei)
    e1, e2 = cp.eps1(enei), cp.eps2(enei)
    exc = off.planewave_potential(cp, POL, DIR, enei, 1)
    st = obem.bem_init(G1, G2, H1, H2, e1, e2, cp.nvec, enei, con01_zero=True)
    phi, a, alpha, De = obem.excitation(st, exc, e1, e2)
    Ax = obem.bem_operator(G1, G2, H1, H2, e1, e2, cp.nvec, enei,
                           sig.sig1[:, None], sig.sig2[:, None], sig.h1[:, :, None], sig.h2[:, :, None])
    b = np.concatenate([phi.ravel(), a.ravel(), alpha.ravel(), De.ravel()])
    r = np.concatenate([x.ravel() for x in Ax]) - b
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-4
    s1, s2, h1, h2, it_ref, rr_ref = obem.iter_solve(G1, G2, H1, H2, e1, e2, cp.nvec, enei, phi, a, alpha, De,
                                                     tol=1e-4, maxit=300)
    assert abs(it[-1] - it_ref) <= 2, (it[-1], it_ref)
    ext_ref = off.extinction(cp, s1[:, None], s2[:, None], h1[:, :, None], h2[:, :, None], enei, POL, DIR)[0]
    assert abs(ext - ext_ref) / abs(ext_ref) < 1e-6, (ext, ext_ref)
    assert rel(sig.sig2, s2) < 1e-6 and rel(sig.h2, h2) < 1e-6


def test_restarted_gmres(cuda):
    cp = sphere()
    bem, sig, ext, _ = _iter(cp, 550.0, precond=None, tol=1e-8, maxit=600, restart=25)
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-8 and it[-1] > 25
    ref = OracleBEM(cp).solve(550.0, POL, DIR)
    assert abs(ext - ref["ext"][0]) / abs(ref["ext"][0]) < 1e-6
