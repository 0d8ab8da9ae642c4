"""The headline workload, pinned to the reference's own result.

The 5768-face gold dimer (2 x trisphere(1444, 40 nm), 2 nm gap on x, water
eps 1.77, Drude gold, x-polarised plane wave along +z, 650 nm) is solved by
the GPU paths and compared with ``tests/golden/dimer_cfg1.npz``, which
``tests/golden/make_golden.py`` wrote by running the unmodified reference
``BEMRet`` (mnpbem/bem/bem_ret.py:1569-1831) on the same mesh:

* the refined-pair counts of the four particle blocks (refinematrix,
  mnpbem/greenfun/refine_utils.py:29-158);
* extinction and scattering: fp64 to 1e-10, the mixed paths (complex64
  factors + FP64 refinement) to 1e-8, the accuracy target of the mixed path;
* checksums of the solution: sum |sig1|, |sig2|, |h1|, |h2| and the first 64
  entries of sig2;
* the H-matrix GMRES path (BEMRetIter(hmatrix=True)) at the same size, to its
  compression tolerance.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

POL = np.array([[1.0, 0, 0]])
DIR = np.array([[0, 0, 1.0]])


def _dimer():
    from mnpbem_b200 import ComParticle, EpsConst, EpsDrude, trisphere
    a, b = trisphere(1444, 40.0), trisphere(1444, 40.0)
    a.shift([-21.0, 0, 0])
    b.shift([21.0, 0, 0])
    return ComParticle([EpsConst(1.77), EpsDrude(9.84, 9.0, 0.067)], [a, b], [[2, 1], [2, 1]], 1, 2,
                       interp="curv")


@pytest.fixture(scope="module")
def cfg1():
    return _dimer(), golden("dimer_cfg1.npz")


def _close(a, b, tol):
    return abs(a - b) <= tol * abs(b)


def test_refined_pairs_per_block(cuda, cfg1):
    import torch
    from mnpbem_b200.greenfun import CompGreenRet
    cp, g = cfg1
    green = CompGreenRet(cp, cp)
    r = green.refined
    half = cp.n // 2
    row = r.row[:r.nref].long()
    col = r.col[:r.nref].long()
    counts = [int(torch.sum((row // half == i) & (col // half == j))) for i in range(2) for j in range(2)]
    assert counts == [int(v) for v in g["nref"]], (counts, g["nref"])


@pytest.mark.parametrize("precision,engine,tol", [("fp64", "simt", 1e-10), ("mixed", "bf16x3", 1e-8),
                                                  ("mixed", "simt", 1e-8)], ids=["fp64", "mixed-bf16x3", "mixed-simt"])
def test_dimer5768_matches_reference(cuda, cfg1, precision, engine, tol):
    from mnpbem_b200 import BEMRet, PlaneWaveRet
    cp, g = cfg1
    bem = BEMRet(cp, precision=precision, engine=engine)
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(cp, float(g["enei"])))
    ext = exc.extinction(sig)
    sca = exc.scattering(sig)[0]
    assert _close(ext, float(g["ext"]), tol), (ext, float(g["ext"]))
    assert _close(sca, float(g["sca"]), tol), (sca, float(g["sca"]))
    stol = 10 * tol
    for key in ("sig1", "sig2", "h1", "h2"):
        assert _close(np.sum(np.abs(getattr(sig, key))), float(g[key + "_abs_sum"]), stol), key
    head = g["sig2_head"]
    assert np.max(np.abs(sig.sig2[:64] - head)) <= stol * np.max(np.abs(head))
    if precision == "mixed":
        assert bem.last_ir[1] <= bem.ir_tol, bem.last_ir


def test_dimer5768_hmatrix_gmres(cuda, cfg1):
    """H-matrix operator (htol 1e-6, cleaf 200) with the complex64 factors as
    preconditioner: the extinction agrees with the reference's dense solve to
    the compression tolerance."""
    from mnpbem_b200 import PlaneWaveRet
    from mnpbem_b200.bem_iter import BEMRetIter
    cp, g = cfg1
    bem = BEMRetIter(cp, hmatrix=True, htol=1e-6, tol=1e-8)
    exc = PlaneWaveRet(POL, DIR)
    sig, bem = bem.solve(exc.potential(cp, float(g["enei"])))
    it, rr, fl = bem.info()
    assert fl[-1] == 0 and rr[-1] <= 1e-8, bem.info()
    assert _close(exc.extinction(sig), float(g["ext"]), 1e-5)
    assert _close(exc.scattering(sig)[0], float(g["sca"]), 1e-5)
