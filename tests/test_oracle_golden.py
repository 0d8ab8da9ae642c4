"""The CPU oracle against golden vectors produced by the reference MNPBEM
(tests/golden/make_golden.py) and against MNPBEM17 MATLAB results."""
import numpy as np
import pytest

from conftest import golden
from meshes import DRUDE_AU, dimer, rel, sphere
from mnpbem_b200.geometry import ComParticle, trisphere
from mnpbem_b200.materials import EpsConst, EpsDrude, EpsValues
from oracle import green as og
from oracle.pipeline import OracleBEM

POL = [[1.0, 0, 0]]
DIR = [[0, 0, 1.0]]


def test_refinement_coefficients_cfg0():
    g = golden("refined_cfg0.npz")
    cp = sphere()
    blocks = og.refine_all(cp)
    b = blocks[0][0]
    assert len(b.rows) == int(g["nref"])
    sel = np.arange(0, len(b.rows), 4)
    np.testing.assert_array_equal(b.rows[sel], g["row"])
    np.testing.assert_array_equal(b.cols[sel], g["col"])
    assert rel(b.g[sel], g["g"]) < 1e-13
    assert rel(b.f[sel], g["f"]) < 1e-13


def test_matrices_and_solution_s60():
    g = golden("matrices_s60.npz")
    cp = ComParticle([EpsConst(1.77), EpsDrude(*DRUDE_AU)], [trisphere(32, 10.0)], [[2, 1]], 1, interp="curv")
    ob = OracleBEM(cp)
    out = ob.solve(float(g["enei"]), POL, DIR, return_state=True)
    for k in ("G1", "G2", "H1", "H2"):
        assert rel(out[k], g[k]) < 1e-13, k
    assert rel(out["state"].Sigma1, g["Sigma1"]) < 1e-11
    assert rel(out["sig1"][:, 0], g["sig1"]) < 1e-11
    assert rel(out["h2"][:, :, 0], g["h2"]) < 1e-11
    assert abs(out["ext"][0] - g["ext"]) / abs(g["ext"]) < 1e-12
    assert abs(out["sca"][0] - g["sca"]) / abs(g["sca"]) < 1e-12


@pytest.mark.slow
def test_spectrum_cfg0():
    g = golden("spectrum_cfg0.npz")
    cp = sphere()
    ob = OracleBEM(cp)
    for i in (0, 20, 40):
        out = ob.solve(float(g["enei"][i]), POL, DIR)
        assert abs(out["ext"][0] - g["ext"][i]) / g["ext"][i] < 1e-11
        assert abs(out["sca"][0] - g["sca"][i]) / g["sca"][i] < 1e-11
        if i == 20:
            assert rel(out["sig2"][:, 0], g["sig2_600"]) < 1e-11
            assert rel(out["h1"][:, :, 0], g["h1_600"]) < 1e-11


def test_dimer_small():
    g = golden("dimer_small.npz")
    cp = dimer()
    ob = OracleBEM(cp)
    b01 = ob.blocks[0][1]
    np.testing.assert_array_equal(b01.rows, g["cross_row"])
    np.testing.assert_array_equal(b01.cols, g["cross_col"])
    assert rel(b01.g, g["cross_g"]) < 1e-13 and rel(b01.f, g["cross_f"]) < 1e-13
    out = ob.solve(620.0, POL, DIR)
    assert abs(out["ext"][0] - g["ext"][1]) / g["ext"][1] < 1e-11
    assert abs(out["sca"][0] - g["sca"][1]) / g["sca"][1] < 1e-11
    assert rel(out["sig1"][:, 0], g["sig1"]) < 1e-10


@pytest.mark.slow
def test_matlab_mnpbem17_tabulated_gold():
    """trisphere(144, 20), tabulated gold: the oracle reproduces MNPBEM17 (MATLAB)
    to the 11 digits stored in the reference's validation CSV."""
    g = golden("matlab_cfg0.npz")
    table = dict(zip(g["enei"], g["eps_gold"]))
    cp = ComParticle([EpsConst(1.0), EpsValues(table)], [trisphere(144, 20.0)], [[2, 1]], 1, interp="curv")
    ob = OracleBEM(cp)
    for i in range(0, 41, 8):
        out = ob.solve(float(g["enei"][i]), POL, DIR)
        assert abs(out["ext"][0] - g["ext"][i]) / g["ext"][i] < 5e-10
        assert abs(out["sca"][0] - g["sca"][i]) / g["sca"][i] < 5e-10


def test_oracle_iterative_matches_mnpbem17():
    """The oracle's unpreconditioned GMRES on the packed 8N system
    (oracle.bem.iter_solve, the reference's BEMRetIter(precond=None) path)
    against MNPBEM17's bemiter extinction of trisphere(144, 20) with tabulated
    gold (validation/08_iterative/sphere/data/ret_matlab.csv).  The packed
    system is ill-conditioned enough that a residual of 1e-9 still leaves
    1e-6 in the extinction, so GMRES runs to 1e-12 here."""
    from oracle import bem as obem
    from oracle import farfield as off
    g = golden("matlab_iter.npz")
    cp = ComParticle([EpsConst(1.0), EpsValues(dict(zip(g["enei"], g["eps_gold"])))], [trisphere(144, 20.0)],
                     [[2, 1]], 1, interp="curv")
    ob = OracleBEM(cp)
    for i in (0, 20, 40):
        enei = float(g["enei"][i])
        G1, G2, H1, H2 = ob.matrices(enei)
        e1, e2 = cp.eps1(enei), cp.eps2(enei)
        st = obem.bem_init(G1, G2, H1, H2, e1, e2, cp.nvec, enei, con01_zero=True)
        phi, a, alpha, De = obem.excitation(st, off.planewave_potential(cp, POL, DIR, enei, 1), e1, e2)
        s1, s2, h1, h2, it, rr = obem.iter_solve(G1, G2, H1, H2, e1, e2, cp.nvec, enei, phi, a, alpha, De,
                                                 tol=1e-12, maxit=3000)
        assert rr <= 1e-12
        ext = off.extinction(cp, s1[:, None], s2[:, None], h1[:, :, None], h2[:, :, None], enei, POL, DIR)[0]
        assert abs(ext - g["ext_iter"][i]) / g["ext_iter"][i] < 1e-7, (i, ext, g["ext_iter"][i])
        assert abs(g["ext_iter"][i] - g["ext_direct"][i]) / g["ext_direct"][i] < 1e-9


def _fixture_solution(g, tag):
    s = [g[tag + "_" + k] for k in ("sig1", "sig2", "h1", "h2")]
    if s[0].ndim == 1:
        s = [s[0][:, None], s[1][:, None], s[2][:, :, None], s[3][:, :, None]]
    return s


@pytest.mark.parametrize("tag,mk", [("dimer", dimer), ("sphere", sphere)])
def test_potential_field_and_cart_derivatives(tag, mk):
    """Oracle CompGreenRet.potential / .field (inside and outside) and the
    Gp / H1p / H2p Green functions against the reference's own BEMRet.potential
    / .field and eval on its solutions (field_potential.npz)."""
    g = golden("field_potential.npz")
    cp = mk()
    ob = OracleBEM(cp)
    enei = float(g[tag + "_enei"])
    s = _fixture_solution(g, tag)
    for io in (1, 2):
        for k, v in zip(("phi", "phip", "a", "ap"), og.potential(cp, ob.blocks, *s, enei, io)):
            ref = g["{}_pot{}_{}".format(tag, io, k)]
            assert rel(np.asarray(v).reshape(ref.shape), ref) < 1e-13, (io, k)
        for k, v in zip("eh", og.field(cp, ob.blocks, *s, enei, io)):
            ref = g["{}_field{}_{}".format(tag, io, k)]
            assert rel(v.reshape(ref.shape), ref) < 1e-13, (io, k)
    for i, j, key in ((0, 0, "H1p"), (1, 1, "H2p"), (1, 1, "Gp"), (0, 0, "Gp")):
        M = og.green_region(cp, ob.blocks, i, j, key, enei)
        nm = "{}_{}{}{}".format(tag, key, i, j)
        assert rel(M[:8], g[nm + "_rows"]) < 1e-13, nm
        assert abs(np.sum(np.abs(M)) - g[nm + "_abssum"]) <= 1e-12 * g[nm + "_abssum"], nm
