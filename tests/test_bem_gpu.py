"""GPU dense BEM (fp64 and mixed + IR) against the CPU oracle and golden vectors."""
import numpy as np
import pytest

from conftest import golden
from meshes import dimer, rel, sphere
from oracle.pipeline import OracleBEM

pytestmark = pytest.mark.gpu

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _run(cp, enei, **kw):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    bem = BEMRet(cp, **kw)
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(cp, enei))
    return bem, sig, exc.extinction(sig), exc.scattering(sig)[0]


@pytest.mark.parametrize("mk,enei", [(sphere, 600.0), (dimer, 620.0)], ids=["sphere284", "dimer568"])
def test_fp64_matches_oracle(cuda, mk, enei):
    cp = mk()
    bem, sig, ext, sca = _run(cp, enei)
    ref = OracleBEM(cp).solve(enei, POL, DIR)
    assert abs(ext - ref["ext"][0]) / abs(ref["ext"][0]) < 1e-10
    assert abs(sca - ref["sca"][0]) / abs(ref["sca"][0]) < 1e-10
    assert rel(sig.sig1, ref["sig1"][:, 0]) < 1e-9
    assert rel(sig.sig2, ref["sig2"][:, 0]) < 1e-9
    assert rel(sig.h1, ref["h1"][:, :, 0]) < 1e-9
    assert rel(sig.h2, ref["h2"][:, :, 0]) < 1e-9


def test_fp64_golden_dimer_small(cuda):
    g = golden("dimer_small.npz")
    cp = dimer()
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    bem = BEMRet(cp)
    exc = PlaneWaveRet(POL, DIR)
    for i, enei in enumerate(g["enei"]):
        sig, bem = bem.solve(exc.potential(cp, float(enei)))
        assert abs(exc.extinction(sig) - g["ext"][i]) / g["ext"][i] < 1e-10
        assert abs(exc.scattering(sig)[0] - g["sca"][i]) / g["sca"][i] < 1e-10


def test_fp64_multi_polarisation(cuda):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp = sphere()
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    bem = BEMRet(cp)
    exc = PlaneWaveRet(pol, dirs)
    sig, _ = bem.solve(exc.potential(cp, 550.0))
    ref = OracleBEM(cp).solve(550.0, pol, dirs)
    ext = exc.extinction(sig)
    assert np.max(np.abs(ext - ref["ext"]) / np.abs(ref["ext"])) < 1e-10
    assert rel(sig.h2, ref["h2"]) < 1e-9


@pytest.mark.parametrize("engine", ["simt", "bf16x3"])
def test_mixed_ir_matches_fp64(cuda, engine):
    cp = dimer()
    _, sig64, ext64, sca64 = _run(cp, 620.0)
    bem, sig, ext, sca = _run(cp, 620.0, precision="mixed", engine=engine)
    it, rr = bem.last_ir[:2]
    assert rr <= 1e-12 and it <= 10, bem.last_ir
    assert abs(ext - ext64) / abs(ext64) < 1e-10
    assert abs(sca - sca64) / abs(sca64) < 1e-10
    assert rel(sig.sig2, sig64.sig2) < 1e-9


def test_operator_residual_of_fp64_solution(cuda):
    """The FP64 dense solution satisfies the full 8N BEM operator (bem200_bem_apply)."""
    import ctypes
    import torch
    from mnpbem_b200 import _native as nat
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    from mnpbem_b200.bem import _excitation_rhs
    cp = sphere()
    enei = 640.0
    bem = BEMRet(cp)
    exc = PlaneWaveRet(POL, DIR)
    e = exc.potential(cp, enei)
    sig, _ = bem.solve(e)
    n = cp.n
    G = bem.g.bem_matrices(enei)
    W1 = torch.as_tensor(np.concatenate([sig.sig1[:, None], sig.h1], axis=1), device="cuda")
    W2 = torch.as_tensor(np.concatenate([sig.sig2[:, None], sig.h2], axis=1), device="cuda")
    _, phi, a, alpha, De = _excitation_rhs(cp, e, enei)
    b = torch.as_tensor(np.concatenate([phi.ravel(), a.ravel(), alpha.ravel(), De.ravel()]), device="cuda")
    r = torch.empty_like(b)
    L = nat.lib()
    scr = torch.empty(int(L.bem200_bem_apply_workspace_size(n, 1)), dtype=torch.uint8, device="cuda")
    e1 = cp.eps1(enei)[0]
    e2 = cp.eps2(enei)[0]
    E1 = (ctypes.c_double * 2)(e1.real, e1.imag)
    E2 = (ctypes.c_double * 2)(e2.real, e2.imag)
    nv = torch.as_tensor(cp.nvec, device="cuda")
    nat.call("bem200_bem_apply", n, 1, nat.ptr(G[0]), nat.ptr(G[1]), nat.ptr(G[2]), nat.ptr(G[3]), 0,
             ctypes.cast(E1, ctypes.c_void_p), ctypes.cast(E2, ctypes.c_void_p), nat.ptr(nv), 2 * np.pi / enei,
             nat.ptr(W1), nat.ptr(W2), nat.ptr(b), nat.ptr(r), nat.ptr(scr), nat.stream_ptr())
    rn = float(torch.max(torch.abs(r)).item())
    bn = float(torch.max(torch.abs(b)).item())
    assert rn / bn < 1e-10


def _cube_needing_exchanges():
    """tricube(12, 60 nm): its Sigma at 600 nm needs one row exchange in a
    partial-pivoting LU (G1, G2 and Delta need none)."""
    from mnpbem_b200 import ComParticle, EpsConst, EpsDrude
    from mnpbem_b200.geometry import tricube
    return ComParticle([EpsConst(1.0), EpsDrude(9.84, 9.0, 0.067)], [tricube(12, 60.0, 0.25, interp="curv")],
                       [[2, 1]], 1, interp="curv")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["dimer", "cube"])
def test_checked_diagonal_pivots_equal_partial_pivoting(cuda, precision, case):
    """pivoting='auto' factors G1, G2, Delta, Sigma without the pivot search
    when partial pivoting would exchange no rows (the dimer at 520 nm) and
    repeats the init with partial pivoting when one needs exchanges (the
    cube's Sigma at 600 nm; the same dimer's Sigma at 620 nm needs one too);
    either way the solution equals pivoting='partial''s."""
    cp, enei = (dimer(), 520.0) if case == "dimer" else (_cube_needing_exchanges(), 600.0)
    a_bem, a_sig, a_ext, a_sca = _run(cp, enei, precision=precision)
    b_bem, b_sig, b_ext, b_sca = _run(cp, enei, precision=precision, pivoting="partial")
    if precision == "fp64":
        assert a_bem.last_pivoting == ("diagonal" if case == "dimer" else "partial")
    elif case == "dimer":
        assert a_bem.last_pivoting == "inverse"
    else:  # the inverses need no pivot order, only their probes' accuracy
        assert a_bem.last_pivoting in ("inverse", "partial")
    assert b_bem.last_pivoting == "partial"
    tol = 1e-12 if precision == "fp64" else 1e-10
    assert abs(a_ext - b_ext) <= tol * abs(b_ext)
    assert abs(a_sca - b_sca) <= tol * abs(b_sca)
    assert rel(a_sig.sig2, b_sig.sig2) < 1e3 * tol


@pytest.mark.parametrize("explicit", [True, False], ids=["inverses", "lu"])
def test_mixed_explicit_inverses_match_lu_factors(cuda, explicit):
    """The mixed solver's two factor forms (explicit complex64 inverses,
    refinement by products; LU factors, refinement by triangular solves)
    reach the FP64 solution on the config-1 family dimer."""
    cp = dimer()
    bem, sig, ext, sca = _run(cp, 520.0, precision="mixed", explicit_inverses=explicit)
    assert bem.last_pivoting == ("inverse" if explicit else "diagonal")
    ref_bem, ref_sig, ref_ext, ref_sca = _run(cp, 520.0, precision="fp64")
    assert abs(ext - ref_ext) <= 1e-10 * abs(ref_ext)
    assert abs(sca - ref_sca) <= 1e-10 * abs(ref_sca)
    assert rel(sig.sig1, ref_sig.sig1) < 1e-8 and rel(sig.h2, ref_sig.h2) < 1e-8
    assert bem.last_ir[0] <= 8
