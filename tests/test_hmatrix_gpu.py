"""Device H-matrix (batched ACA compression + two-phase matvec) against the
oracle ACA and the dense matrix; BEMRetIter(hmatrix=True) against the direct
FP64 solve."""
import numpy as np
import pytest

from meshes import DRUDE_AU, dimer, rel
from mnpbem_b200.geometry import ComParticle, trisphere
from mnpbem_b200.hmatrix import ClusterTree, HMatrixGPU, block_partition, make_kaware_fadmiss, particle_index
from mnpbem_b200.materials import EpsConst, EpsDrude
from oracle import hmatrix as oh
from oracle.pipeline import OracleBEM

pytestmark = pytest.mark.gpu
ENEI = 600.0
POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _case(tag):
    if tag == "s":
        cp = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE_AU)], [trisphere(144, 20.0)], [[2, 1]], 1, interp="curv")
        return cp, 32, 1.0
    return dimer(), 64, 2.5


def _reconstruct(h):
    """Dense particle-order matrix from the device H-matrix."""
    n = h.n
    t = h.tree
    D, U, V = h.D.cpu().numpy(), h.U.cpu().numpy(), h.V.cpu().numpy()
    out = np.zeros((n, n), dtype=complex)
    for b, (r0, m, c0, nb) in enumerate(h._db):
        o = h._doff_h[b]
        out[r0:r0 + m, c0:c0 + nb] = D[o:o + m * nb].reshape(m, nb)
    for b, (r0, m, c0, nb) in enumerate(h._lb):
        kc, r = int(h._kcap[b]), int(h.ranks[b])
        Ub = U[h._uoff_h[b]:h._uoff_h[b] + m * kc].reshape(m, kc)[:, :r]
        Vb = V[h._voff_h[b]:h._voff_h[b] + nb * kc].reshape(nb, kc)[:, :r]
        out[r0:r0 + m, c0:c0 + nb] = Ub @ Vb.T
    p2c = t.ind[:, 1]
    return out[np.ix_(p2c, p2c)]


@pytest.mark.parametrize("tag", ["s", "d"])
def test_gpu_aca_matches_oracle(cuda, tag):
    import torch
    cp, cleaf, eta = _case(tag)
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    dense, low = block_partition(t, make_kaware_fadmiss(2 * np.pi / ENEI, eta0=eta))
    G1 = OracleBEM(cp).matrices(ENEI)[0]
    full_ref, ranks_ref = oh.hmatrix_full(t, dense, low, G1, htol=1e-6, kmax=100)
    h = HMatrixGPU(t, dense, low, htol=1e-6, kmax=100).compress(torch.as_tensor(G1, device="cuda"))
    np.testing.assert_array_equal(h.ranks, ranks_ref)
    full = _reconstruct(h)
    # same factors up to rounding: the reconstructions agree far below the ACA error
    assert np.linalg.norm(full - full_ref) / np.linalg.norm(G1) < 1e-11
    # stored elements / n^2, the reference's HMatrix.compression formula (can exceed 1
    # for small blocks whose rank is large against their size)
    nel = sum(m * nb for _, m, _, nb in h._db) + sum((m + nb) * r for (_, m, _, nb), r in zip(h._lb, ranks_ref))
    assert abs(h.compression() - nel / cp.n ** 2) < 1e-12


@pytest.mark.parametrize("tag", ["s", "d"])
@pytest.mark.parametrize("w", [1, 8, 16])
def test_gpu_hmatrix_matvec(cuda, tag, w):
    import torch
    cp, cleaf, eta = _case(tag)
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    dense, low = block_partition(t, make_kaware_fadmiss(2 * np.pi / ENEI, eta0=eta))
    G1 = OracleBEM(cp).matrices(ENEI)[0]
    h = HMatrixGPU(t, dense, low, htol=1e-6, kmax=100).compress(torch.as_tensor(G1, device="cuda"))
    full = _reconstruct(h)
    rng = np.random.default_rng(w)
    x = rng.standard_normal((cp.n, w)) + 1j * rng.standard_normal((cp.n, w))
    c2p = t.ind[:, 0]
    xc = torch.as_tensor(np.ascontiguousarray(x[c2p]), device="cuda")
    yc = torch.empty_like(xc)
    h.matvec(xc, yc, w)
    y = np.empty_like(x)
    y[c2p] = yc.cpu().numpy()
    assert rel(y, full @ x) < 1e-13
    assert rel(y, G1 @ x) < 1e-5
    # the one-CTA-per-block product agrees (FP64 atomics: summation order differs)
    yb = torch.empty_like(xc)
    h.matvec_per_block(xc, yb, w)
    assert rel(yb.cpu().numpy(), yc.cpu().numpy()) < 1e-13


@pytest.mark.parametrize("mk", ["sphere", "dimer"])
def test_bem_iter_hmatrix(cuda, mk):
    """BEMRetIter(hmatrix=True): H-matrix operator, dense complex64 factors as
    preconditioner, converged to 1e-10 -- ext within the H-matrix tolerance of
    the direct FP64 solve."""
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.bem_iter import BEMRetIter
    if mk == "sphere":
        cp, cleaf, eta = _case("s")
    else:
        cp, cleaf, eta = _case("d")
    bem = BEMRetIter(cp, hmatrix=True, cleaf=cleaf, eta=eta, htol=1e-6, tol=1e-10)
    exc = PlaneWaveRet(POL, DIR)
    sig, _ = bem.solve(exc.potential(cp, ENEI))
    ext = exc.extinction(sig)
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-10
    ref = OracleBEM(cp).solve(ENEI, POL, DIR)
    assert abs(ext - ref["ext"][0]) / abs(ref["ext"][0]) < 1e-5
    comp = bem._hmat.compression()
    assert all(c > 0 for c in comp)


@pytest.mark.parametrize("tag", ["s", "d"])
def test_green_fill_matches_dense_fill(cuda, tag):
    """bem200_hmat_compress_green (entries on demand, no n x n matrix) against
    compressing the assembled dense matrices, for G1, G2, H1, H2."""
    from mnpbem_b200.greenfun import CompGreenRet
    cp, cleaf, eta = _case(tag)
    g = CompGreenRet(cp, cp)
    mats = g.bem_matrices(ENEI, dtype="c128")
    t = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=particle_index(cp))
    dense, low = block_partition(t, make_kaware_fadmiss(2 * np.pi / ENEI, eta0=eta))
    for which, M in enumerate(mats):
        hd = HMatrixGPU(t, dense, low, htol=1e-6, kmax=100).compress(M)
        hg = HMatrixGPU(t, dense, low, htol=1e-6, kmax=100).compress_green(g, ENEI, which)
        # dense leaves: the same entries as the assembly kernels, to rounding
        assert rel(hg.D.cpu().numpy(), hd.D.cpu().numpy()) < 1e-13, which
        assert np.mean(hg.ranks == hd.ranks) > 0.9, which
        Md = M.cpu().numpy()
        fg = _reconstruct(hg)
        assert np.linalg.norm(fg - _reconstruct(hd)) / np.linalg.norm(Md) < 1e-5, which
        assert np.linalg.norm(fg - Md) / np.linalg.norm(Md) < 1e-5, which


def test_bem_iter_hmatrix_green_fill(cuda):
    """BEMRetIter(hmatrix=True) with the on-demand fill, unpreconditioned and
    preconditioned, against the fill from the dense matrices."""
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.bem_iter import BEMRetIter
    cp, cleaf, eta = _case("d")
    exc = PlaneWaveRet(POL, DIR)
    ext = {}
    for fill in ("green", "dense"):
        for precond in ("hmat", None):
            bem = BEMRetIter(cp, hmatrix=True, cleaf=cleaf, eta=eta, htol=1e-6, tol=1e-9, maxit=400,
                             precond=precond, hmat_fill=fill)
            sig, _ = bem.solve(exc.potential(cp, ENEI))
            it, rr, fl = bem.info()
            assert fl[-1] == 0 and rr[-1] <= 1e-9, (fill, precond, it, rr)
            ext[fill, precond] = exc.extinction(sig)
    for precond in ("hmat", None):
        assert abs(ext["green", precond] - ext["dense", precond]) / abs(ext["dense", precond]) < 1e-6
    ref = OracleBEM(cp).solve(ENEI, POL, DIR)["ext"][0]
    assert abs(ext["green", None] - ref) / abs(ref) < 1e-5
