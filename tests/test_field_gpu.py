"""Potentials and fields of a solution at the faces on the GPU (reference
BEMRet.potential / BEMRet.field, mnpbem/bem/bem_ret.py:1833-1895, through
CompGreenRet.potential / .field, mnpbem/greenfun/compgreen_ret.py:912-1038),
and the Cartesian-derivative Green functions Gp / H1p / H2p
(mnpbem/greenfun/greenret_refined.py:812-864).

Inputs are the reference's own solutions stored in field_potential.npz; the
outputs are compared with the reference's results to 1e-10.  At the
5768-face size, where no CPU result is stored, the on-the-fly products are
checked against the product of the assembled matrices (a size-independent
identity: the fused kernel must equal G x sigma computed from the stored
matrix)."""
import numpy as np
import pytest

from conftest import golden
from meshes import dimer, rel, sphere

pytestmark = pytest.mark.gpu


def _sig(cp, g, tag):
    from mnpbem_b200.planewave import CompStruct
    return CompStruct(cp, float(g[tag + "_enei"]), **{k: g[tag + "_" + k] for k in ("sig1", "sig2", "h1", "h2")})


@pytest.mark.parametrize("tag,mk", [("dimer", dimer), ("sphere", sphere)])
def test_potential_and_field_match_reference(cuda, tag, mk):
    from mnpbem_b200 import BEMRet
    g = golden("field_potential.npz")
    cp = mk()
    bem = BEMRet(cp)
    sig = _sig(cp, g, tag)
    for io in (1, 2):
        pot = bem.potential(sig, io)
        for k, name in (("phi", "phi{}"), ("phip", "phi{}p"), ("a", "a{}"), ("ap", "a{}p")):
            ref = g["{}_pot{}_{}".format(tag, io, k)]
            got = np.asarray(getattr(pot, name.format(io)))
            assert got.shape == ref.shape, (io, k, got.shape, ref.shape)
            assert rel(got, ref) < 1e-10, (io, k, rel(got, ref))
        f = bem.field(sig, io)
        for k in "eh":
            ref = g["{}_field{}_{}".format(tag, io, k)]
            got = np.asarray(getattr(f, k))
            assert got.shape == ref.shape, (io, k, got.shape, ref.shape)
            assert rel(got, ref) < 1e-10, (io, k, rel(got, ref))


@pytest.mark.parametrize("tag,mk", [("dimer", dimer), ("sphere", sphere)])
def test_cart_derivative_green_functions(cuda, tag, mk):
    from mnpbem_b200.greenfun import CompGreenRet
    g = golden("field_potential.npz")
    cp = mk()
    green = CompGreenRet(cp, cp)
    enei = float(g[tag + "_enei"])
    for i, j, key in ((0, 0, "H1p"), (1, 1, "H2p"), (1, 1, "Gp"), (0, 0, "Gp")):
        M = green.eval(i, j, key, enei)
        nm = "{}_{}{}{}".format(tag, key, i, j)
        assert M.shape == (cp.n, 3, cp.n)
        assert rel(M[:8], g[nm + "_rows"]) < 1e-11, nm  # FP64 quadrature sums in another order: ~2e-12
        assert abs(np.sum(np.abs(M)) - g[nm + "_abssum"]) <= 1e-11 * g[nm + "_abssum"], nm
    assert green.eval(1, 0, "H1p", enei) == 0  # no region pair connects: the reference's int 0


@pytest.mark.slow
def test_fused_products_equal_assembled_products_5768(cuda):
    """5768-face dimer: the on-the-fly potential and field equal the products
    of the assembled G / H / H1p matrices with a seeded solution."""
    import torch
    from mnpbem_b200 import ComParticle, EpsConst, EpsDrude, trisphere
    from mnpbem_b200.greenfun import CompGreenRet
    from mnpbem_b200.planewave import CompStruct
    a, b = trisphere(1444, 40.0), trisphere(1444, 40.0)
    a.shift([-21.0, 0, 0])
    b.shift([21.0, 0, 0])
    cp = ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)], [a, b], [[2, 1], [2, 1]], 1, 2, interp="curv")
    n, enei = cp.n, 650.0
    rng = np.random.default_rng(3)

    def c(*shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    sig = CompStruct(cp, enei, sig1=c(n, 2), sig2=c(n, 2), h1=c(n, 3, 2), h2=c(n, 3, 2))
    green = CompGreenRet(cp, cp)
    dev = torch.device("cuda")
    t = {k: torch.as_tensor(getattr(sig, k), device=dev) for k in ("sig1", "sig2", "h1", "h2")}
    pot = green.potential(sig, 1)
    G0 = green.eval(0, 0, "G", enei, as_tensor=True)
    H0 = green.eval(0, 0, "H1", enei, as_tensor=True)
    G1 = green.eval(0, 1, "G", enei, as_tensor=True)
    assert isinstance(G1, int) and G1 == 0  # the inside of one sphere sees nothing of the other's outside
    phi = (G0 @ t["sig1"]).cpu().numpy()
    ap = torch.einsum("ij,jcp->icp", H0, t["h1"]).cpu().numpy()
    assert rel(pot.phi1, phi) < 1e-11 and rel(pot.a1p, ap) < 1e-11
    del G0, H0
    f = green.field(sig, 2)
    G = green.eval(1, 1, "G", enei, as_tensor=True)
    e = 2j * np.pi / enei * torch.einsum("ij,jcp->icp", G, t["h2"])
    del G
    P = green.eval(1, 1, "H2p", enei, as_tensor=True)
    e = (e - torch.einsum("icj,jp->icp", P, t["sig2"])).cpu().numpy()
    hx = (torch.einsum("ij,jp->ip", P[:, 1], t["h2"][:, 2]) - torch.einsum("ij,jp->ip", P[:, 2], t["h2"][:, 1]))
    assert rel(f.e, e) < 1e-11
    assert rel(f.h[:, 0], hx.cpu().numpy()) < 1e-11
